// Device pieces of the Fourier response generators shared by the kernel-bank
// generation (jerk_bank.cu) and the candidate polishing (jerk_polish.cu).
#pragma once

#include <cuda_runtime.h>

#include <cmath>

namespace jerk {

// Fresnel integrals C(x) = int_0^x cos(pi t^2/2) dt, S(x) = int_0^x sin(pi t^2/2) dt.
// |x| < 1.5: the power series of int_0^x exp(i pi t^2/2) dt,
//   sum_k (i pi/2)^k x^(2k+1) / (k! (2k+1));
// otherwise C + iS = (1+i)/2 * erf(sqrt(pi)/2 (1-i) x), with erfc from its
// even continued fraction (denominators 1 - i pi x^2 + 4k, numerators
// -(2k-1)(2k)), evaluated by the modified Lentz method.
static __device__ void fresnel(double x, double *S, double *C)
{
    const double ax = fabs(x);
    double c = 0.0, s = 0.0;
    if (ax < 1.5) {
        const double p = 0.5 * M_PI * ax * ax;
        double ft = ax;
        for (int k = 0; k < 60; k++) {
            const double term = ft / (2 * k + 1);
            switch (k & 3) {
            case 0: c += term; break;
            case 1: s += term; break;
            case 2: c -= term; break;
            default: s -= term; break;
            }
            ft *= p / (k + 1);
            if (ft < 1e-18 * (fabs(c) + fabs(s)))
                break;
        }
    } else {
        const double pix2 = M_PI * ax * ax;
        double br = 1.0, bi = -pix2;
        double ccr = 1e300, cci = 0.0;
        // d = h = 1 / b
        double den = br * br + bi * bi;
        double dr = br / den, di = -bi / den;
        double hr = dr, hi = di;
        int n = -1;
        for (int k = 2; k < 300; k++) {
            n += 2;
            const double a = -(double)n * (n + 1);
            br += 4.0;
            // d = 1 / (a d + b)
            double tr = a * dr + br, ti = a * di + bi;
            den = tr * tr + ti * ti;
            dr = tr / den;
            di = -ti / den;
            // cc = b + a / cc
            den = ccr * ccr + cci * cci;
            const double qr = a * ccr / den, qi = -a * cci / den;
            ccr = br + qr;
            cci = bi + qi;
            // del = cc d ; h = h del
            const double er = ccr * dr - cci * di, ei = ccr * di + cci * dr;
            const double nhr = hr * er - hi * ei, nhi = hr * ei + hi * er;
            hr = nhr;
            hi = nhi;
            if (fabs(er - 1.0) + fabs(ei) < 1e-16)
                break;
        }
        // h = (ax - i ax) h
        const double h2r = ax * hr + ax * hi, h2i = ax * hi - ax * hr;
        double sn, cs;
        sincos(0.5 * pix2, &sn, &cs);
        // (cos + i sin) h
        const double mr = cs * h2r - sn * h2i, mi = cs * h2i + sn * h2r;
        // (0.5 + 0.5 i)(1 - m)
        const double ur = 1.0 - mr, ui = -mi;
        c = 0.5 * ur - 0.5 * ui;
        s = 0.5 * ur + 0.5 * ui;
    }
    if (x < 0.0) {
        c = -c;
        s = -s;
    }
    *C = c;
    *S = s;
}


// value numbers ii of the raw response (src/responses.c), then placement:
// raw index ii < numkern/2 goes to fftlen - numkern/2 + ii, the rest to
// ii - numkern/2 (src/corr_prep.c:92-114)
static __device__ __forceinline__ long long placed(int ii, int numkern, int fftlen)
{
    const int half = numkern / 2;
    return ii < half ? (long long)(fftlen - half + ii) : (long long)(ii - half);
}

}  // namespace jerk
