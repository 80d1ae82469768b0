/*
 * Double-precision mixed-radix complex FFT (see mixfft.h).
 * TEST INFRASTRUCTURE ONLY: used by the oracle and the FFTW stand-in.
 */
#include "mixfft.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct mixfft_plan {
    int n;
    int sign;
    int nfac;
    int fac[64];
    double *tw; /* tw[2k], tw[2k+1] = cos, sin of sign*2*pi*k/n */
};

mixfft_plan *mixfft_create(int n, int sign)
{
    mixfft_plan *p;
    int m, f;

    if (n < 1)
        return NULL;
    p = (mixfft_plan *)calloc(1, sizeof(*p));
    if (!p)
        return NULL;
    p->n = n;
    p->sign = sign < 0 ? -1 : 1;
    m = n;
    while (m > 1) {
        if (m % 4 == 0)
            f = 4;
        else if (m % 2 == 0)
            f = 2;
        else if (m % 3 == 0)
            f = 3;
        else if (m % 5 == 0)
            f = 5;
        else {
            for (f = 7; f * f <= m; f += 2)
                if (m % f == 0)
                    break;
            if (f * f > m)
                f = m;
        }
        p->fac[p->nfac++] = f;
        m /= f;
    }
    if (p->nfac == 0)
        p->fac[p->nfac++] = 1;
    p->tw = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    if (!p->tw) {
        free(p);
        return NULL;
    }
    for (int k = 0; k < n; k++) {
        /* exact values on the axes keep the table symmetric */
        double ang = p->sign * 2.0 * M_PI * (double)k / (double)n;
        p->tw[2 * k] = cos(ang);
        p->tw[2 * k + 1] = sin(ang);
        if (4 * (long)k == n) {
            p->tw[2 * k] = 0.0;
            p->tw[2 * k + 1] = p->sign;
        } else if (2 * (long)k == n) {
            p->tw[2 * k] = -1.0;
            p->tw[2 * k + 1] = 0.0;
        } else if (4 * (long)k == 3 * (long)n) {
            p->tw[2 * k] = 0.0;
            p->tw[2 * k + 1] = -p->sign;
        }
    }
    return p;
}

void mixfft_destroy(mixfft_plan *p)
{
    if (!p)
        return;
    free(p->tw);
    free(p);
}

int mixfft_size(const mixfft_plan *p) { return p->n; }

/* out[0..n) = DFT_n of in[0], in[stride], ...  (complex, interleaved) */
static void rec(const mixfft_plan *P, double *out, const double *in, int n,
                long stride, const int *fac)
{
    const int p = fac[0];
    const int m = n / p;
    const long twstep = P->n / n;
    const long pstep = P->n / p;
    const double *tw = P->tw;

    if (m == 1) {
        for (int q = 0; q < p; q++) {
            out[2 * q] = in[2 * q * stride];
            out[2 * q + 1] = in[2 * q * stride + 1];
        }
    } else {
        for (int q = 0; q < p; q++)
            rec(P, out + 2L * q * m, in + 2L * q * stride, m, stride * p, fac + 1);
    }
    if (p == 1)
        return;

    double tbuf[2 * 64];
    double *t = p <= 64 ? tbuf : (double *)malloc(sizeof(double) * 2 * (size_t)p);
    double ybuf[2 * 64];
    double *y = p <= 64 ? ybuf : (double *)malloc(sizeof(double) * 2 * (size_t)p);

    for (int k = 0; k < m; k++) {
        /* twiddle: t_q = F_q[k] * w_n^(q*k) */
        t[0] = out[2L * k];
        t[1] = out[2L * k + 1];
        for (int q = 1; q < p; q++) {
            const long idx = (long)q * k * twstep;
            const double wr = tw[2 * idx], wi = tw[2 * idx + 1];
            const double xr = out[2L * (q * m + k)], xi = out[2L * (q * m + k) + 1];
            t[2 * q] = xr * wr - xi * wi;
            t[2 * q + 1] = xr * wi + xi * wr;
        }
        if (p == 2) {
            out[2L * k] = t[0] + t[2];
            out[2L * k + 1] = t[1] + t[3];
            out[2L * (m + k)] = t[0] - t[2];
            out[2L * (m + k) + 1] = t[1] - t[3];
        } else if (p == 4) {
            /* w_4 = sign * i */
            const double s = P->sign;
            const double ar = t[0] + t[4], ai = t[1] + t[5];
            const double br = t[0] - t[4], bi = t[1] - t[5];
            const double cr = t[2] + t[6], ci = t[3] + t[7];
            const double dr = t[2] - t[6], di = t[3] - t[7];
            /* w * d = s * (-di + i dr) */
            const double wdr = -s * di, wdi = s * dr;
            out[2L * k] = ar + cr;
            out[2L * k + 1] = ai + ci;
            out[2L * (m + k)] = br + wdr;
            out[2L * (m + k) + 1] = bi + wdi;
            out[2L * (2 * m + k)] = ar - cr;
            out[2L * (2 * m + k) + 1] = ai - ci;
            out[2L * (3 * m + k)] = br - wdr;
            out[2L * (3 * m + k) + 1] = bi - wdi;
        } else {
            for (int s = 0; s < p; s++) {
                double yr = 0.0, yi = 0.0;
                for (int q = 0; q < p; q++) {
                    const long idx = (long)((q * s) % p) * pstep;
                    const double wr = tw[2 * idx], wi = tw[2 * idx + 1];
                    yr += t[2 * q] * wr - t[2 * q + 1] * wi;
                    yi += t[2 * q] * wi + t[2 * q + 1] * wr;
                }
                y[2 * s] = yr;
                y[2 * s + 1] = yi;
            }
            for (int s = 0; s < p; s++) {
                out[2L * (s * m + k)] = y[2 * s];
                out[2L * (s * m + k) + 1] = y[2 * s + 1];
            }
        }
    }
    if (t != tbuf)
        free(t);
    if (y != ybuf)
        free(y);
}

void mixfft_exec(const mixfft_plan *p, const double *in, double *out)
{
    rec(p, out, in, p->n, 1, p->fac);
}
