/*
 * ORACLE: a CPU restatement of the reference's jerk-search hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load this library, and only as the
 * checker.  The product never links or calls it.
 *
 * It works on explicit arrays (spectrum, kernel bank, search geometry), so it
 * can be fed exactly the inputs the CUDA path gets.  Arithmetic follows the
 * reference step for step; the differences are deliberate and stated:
 *   - the forward FFT of the data chunk, the correlation multiply and the
 *     inverse FFT are computed in double precision (the reference uses float
 *     FFTW), so the oracle's powers are the float rounding of a
 *     double-precision correlation;
 *   - everything on the integer/index side is bit-exact with the reference.
 *
 * Reference functions restated (file:line in the reference project):
 *   calc_required_r/z/w, index_from_r/z/w   src/accel_utils.c:54-97
 *   NEAREST_INT                            src/accel_utils.c:36
 *   calc_fftlen                            src/accel_utils.c:137-149
 *   init_subharminfo (zmax/wmax, dims)     src/accel_utils.c:199-234
 *   create_accelobs sizing                 src/accel_utils.c:1795-2004
 *   get_fourier_amplitudes                 src/accel_utils.c:1058-1092
 *   subharm_fderivs_vol                    src/accel_utils.c:1094-1293
 *   add_ffdotpows                          src/accel_utils.c:1356-1377
 *   search_ffdotpows                       src/accel_utils.c:1507-1555
 *   insert_new_accelcand                   src/accel_utils.c:382-480
 *   accelsearch main loop                  src/accelsearch.c:183-223
 *   median (order statistic (n-1)/2)       src/median.c:12-69
 *   spread_no_pad                          src/corr_prep.c:62-74
 *   next_good_fftlen, fftlen_from_kernwidth src/corr_prep.c:3-35
 *   z_resp_halfwidth, w_resp_halfwidth     src/responses.c:27-84
 *   candidate_sigma, chi2_logp2,
 *   equivalent_gaussian_sigma2,
 *   extended_equiv_gaussian_sigma,
 *   log_asymtotic_incomplete_gamma/gamma   src/characteristics.c:400-668
 *   cdfchi2 / gratio2 (integer a)          src/dcdflib.c:2336-2476
 *   power_for_sigma                        src/characteristics.c:670-705
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "mixfft.h"

#define ACCEL_NUMBETWEEN 2
#define ACCEL_DR 0.5
#define ACCEL_RDR 2
#define ACCEL_DZ 2
#define ACCEL_RDZ 0.5
#define ACCEL_DW 20
#define ACCEL_RDW 0.05
#define ACCEL_CLOSEST_R 15.0
#define DBLCORRECT 1e-14
#define NUMFINTBINS 16
#define NEAREST_INT(x) (int)((x) < 0 ? (x)-0.5 : (x) + 0.5)

/* ------------------------------------------------------------------ */
/* Geometry                                                            */

typedef struct orc_geom {
    long long numbins;     /* complex bins in the spectrum */
    long long lobin;       /* lowest bin present in the file */
    long long highestbin;  /* highest bin searched */
    double rlo;            /* first fundamental r searched */
    double zlo;            /* -zmax */
    double wlo;            /* -wmax */
    int corr_uselen;
    int numz;              /* fundamental numz (obs->numz) */
    int numharmstages;
    int norm_type;         /* 0 = block median, 1 = local power (-locpow) */
    double nph;            /* > 0: photon normalisation */
    float powcut[6];
    long long numindep[6];
} orc_geom;

typedef struct orc_sub {
    int numharm, harmnum;
    int numz, numw;        /* numkern_zdim, numkern_wdim */
    int fftlen;
    int halfwidth;         /* kern[0][0].kern_half_width */
    const float *kern;     /* [numw][numz][fftlen] complex64 */
} orc_sub;

typedef struct orc_cand {
    float power, sigma;
    int numharm;
    double r, z, w;
} orc_cand;

static double calc_required_r(double harm_fract, double rfull)
{
    return rint(ACCEL_RDR * rfull * harm_fract) * ACCEL_DR;
}

static int calc_required_z(double harm_fract, double zfull)
{
    return NEAREST_INT(ACCEL_RDZ * zfull * harm_fract) * ACCEL_DZ;
}

static int calc_required_w(double harm_fract, double wfull)
{
    return NEAREST_INT(ACCEL_RDW * wfull * harm_fract) * ACCEL_DW;
}

static int index_from_r(double r, double lor) { return (int)((r - lor) * ACCEL_RDR + DBLCORRECT); }
static int index_from_z(double z, double loz) { return (int)((z - loz) * ACCEL_RDZ + DBLCORRECT); }
static int index_from_w(double w, double low) { return (int)((w - low) * ACCEL_RDW + DBLCORRECT); }

int orc_calc_required_z(double hf, double z) { return calc_required_z(hf, z); }
int orc_calc_required_w(double hf, double w) { return calc_required_w(hf, w); }
double orc_calc_required_r(double hf, double r) { return calc_required_r(hf, r); }

int orc_z_resp_halfwidth(double z)
{
    return (int)(0.5 * 1.1 * fabs(z)) + NUMFINTBINS; /* LOWACC */
}

int orc_w_resp_halfwidth(double z, double w)
{
    double r0, r1, maxdev, u_ext;
    if (fabs(w) < 1.0e-7)
        return orc_z_resp_halfwidth(z);
    r0 = 0.5 * (w / 6.0 - z);
    r1 = 0.5 * (w / 6.0 + z);
    maxdev = fabs(r0) > fabs(r1) ? fabs(r0) : fabs(r1);
    u_ext = 0.5 - z / w;
    if (u_ext > 0.0 && u_ext < 1.0) {
        double z0 = z - w / 2.0;
        double r_ext = 0.5 * w * u_ext * u_ext + z0 * u_ext + r0;
        maxdev = fabs(r_ext) > maxdev ? fabs(r_ext) : maxdev;
    }
    return (int)(1.1 * maxdev) + NUMFINTBINS; /* LOWACC */
}

static long long next2_to_n(long long x)
{
    long long n = 1;
    while (n < x)
        n <<= 1;
    return n;
}

int orc_next_good_fftlen(int N)
{
    static const int fftlens[17] = {128, 192, 256, 384, 512, 768, 1024, 1280, 2048,
                                    4096, 5120, 7680, 10240, 12288, 15360, 16384, 25600};
    int ii = 0;
    if (N <= fftlens[0])
        return fftlens[0];
    if (N > fftlens[16])
        return (int)next2_to_n(N);
    while (N > fftlens[ii])
        ii++;
    return fftlens[ii];
}

int orc_fftlen_from_kernwidth(int kernwidth)
{
    if (kernwidth < 6) return 128;
    else if (kernwidth < 52) return 256;
    else if (kernwidth < 67) return 512;
    else if (kernwidth < 378) return 1024;
    else if (kernwidth < 664) return 2048;
    else if (kernwidth < 1672) return 4096;
    else if (kernwidth < 3015) return 10240;
    else if (kernwidth < 3554) return 15360;
    else if (kernwidth < 6000) return 25600;
    else return (int)next2_to_n(kernwidth * 5);
}

/* Sizing of create_accelobs for (zmax, wmax) already rounded to even / a
 * multiple of 20.  out: maxkernlen, fftlen, corr_uselen. */
void orc_obs_sizes(int zmax, int wmax, int *out)
{
    int maxkernlen = 2 * ACCEL_NUMBETWEEN * orc_w_resp_halfwidth(zmax, wmax);
    int fftlen = orc_fftlen_from_kernwidth(maxkernlen);
    int uselen;
    if (fftlen < 2048)
        fftlen = 2048;
    uselen = fftlen - maxkernlen;
    if (uselen % ACCEL_RDR)
        uselen = uselen / ACCEL_RDR * ACCEL_RDR;
    out[0] = maxkernlen;
    out[1] = fftlen;
    out[2] = uselen;
}

/* init_subharminfo dimensions + calc_fftlen.  out: zmax, wmax, numz, numw,
 * fftlen, halfwidth (of kern[0][0], i.e. z = -zmax, w = -wmax). */
void orc_sub_sizes(int numharm, int harmnum, int zmax, int wmax, int corr_uselen,
                   int fund_fftlen, int *out)
{
    double hf = (double)harmnum / (double)numharm;
    int szmax = calc_required_z(hf, zmax);
    int swmax = calc_required_w(hf, wmax);
    int fftlen;
    if (numharm == 1 && harmnum == 1) {
        fftlen = fund_fftlen;
    } else {
        int bins_needed = (int)ceil(corr_uselen * hf) + 2;
        int end_effects = 2 * ACCEL_NUMBETWEEN *
                          orc_w_resp_halfwidth(calc_required_z(hf, zmax),
                                               calc_required_w(hf, wmax));
        fftlen = orc_next_good_fftlen(bins_needed + end_effects);
    }
    out[0] = szmax;
    out[1] = swmax;
    out[2] = (szmax / ACCEL_DZ) * 2 + 1;
    out[3] = (swmax / ACCEL_DW) * 2 + 1;
    out[4] = fftlen;
    out[5] = orc_w_resp_halfwidth((double)-szmax, (double)-swmax);
}

/* ------------------------------------------------------------------ */
/* Statistics (candidate sigma, power cutoff)                          */

/* A&S 6.5.32 series of src/characteristics.c:420-439; for integer a it
 * terminates after a-1 terms. */
static double log_asymtotic_incomplete_gamma(double a, double z)
{
    double x = 1.0, newxpart = 1.0, term = 1.0;
    int ii = 1;
    while (fabs(newxpart) > 1e-15) {
        term *= (a - ii);
        newxpart = term / pow(z, ii);
        x += newxpart;
        ii += 1;
    }
    return (a - 1.0) * log(z) - z + log(x);
}

/* A&S 6.1.41 Stirling series, four terms (src/characteristics.c:441-453). */
static double log_asymtotic_gamma(double z)
{
    double x, y;
    x = (z - 0.5) * log(z) - z + 0.91893853320467267;
    y = 1.0 / (z * z);
    x += (((-5.9523809523809529e-4 * y + 7.9365079365079365079365e-4) * y -
           2.7777777777777777777778e-3) * y + 8.3333333333333333333333e-2) / z;
    return x;
}

/* Upper regularised incomplete gamma Q(a, x) for the integer a = numsum that
 * the search uses: Q = exp(-x) * sum_{n<a} x^n / n!, the closed form that the
 * reference's gratio2 evaluates for integer a. */
static double q_gamma_int(int a, double x)
{
    double sum, t;
    if (x <= 0.0)
        return 1.0;
    sum = t = exp(-x);
    for (int n = 1; n < a; n++) {
        t = t * x / n;
        sum += t;
    }
    return sum;
}

/* Natural log of the upper tail of chi^2 (src/characteristics.c:588-628). */
static double chi2_logp2(double chi2, double dof)
{
    if (chi2 <= 0.0)
        return -INFINITY;
    if (chi2 / dof > 15.0 || (dof > 150 && chi2 / dof > 6.0))
        return log_asymtotic_incomplete_gamma(0.5 * dof, 0.5 * chi2) -
               log_asymtotic_gamma(0.5 * dof);
    return log(q_gamma_int((int)(0.5 * dof + 0.5), 0.5 * chi2));
}

/* Normal quantile: x with Phi(x) = p, for 0 < p < 1, by a bisection bracket
 * refined with Newton steps on erfc (full double precision). */
static double norm_quantile_upper(double q)
{
    /* returns x with Q(x) = 1 - Phi(x) = q */
    double lo = -40.0, hi = 40.0, x = 0.0;
    for (int it = 0; it < 200; it++) {
        x = 0.5 * (lo + hi);
        double qx = 0.5 * erfc(x / M_SQRT2);
        if (qx > q)
            lo = x;
        else
            hi = x;
        if (hi - lo < 1e-15 * (fabs(x) + 1.0))
            break;
    }
    for (int it = 0; it < 3; it++) {
        double qx = 0.5 * erfc(x / M_SQRT2);
        double dens = exp(-0.5 * x * x) / sqrt(2.0 * M_PI);
        if (dens <= 0.0)
            break;
        x += (qx - q) / dens;
    }
    return x;
}

/* A&S 26.2.23 on log p (src/characteristics.c:400-418). */
static double extended_equiv_gaussian_sigma(double logp)
{
    double t, num, denom;
    t = sqrt(-2.0 * logp);
    num = 2.515517 + t * (0.802853 + t * 0.010328);
    denom = 1.0 + t * (1.432788 + t * (0.189269 + t * 0.001308));
    return t - num / denom;
}

static double equivalent_gaussian_sigma2(double logp)
{
    double x;
    if (logp < -600.0) {
        x = extended_equiv_gaussian_sigma(logp);
    } else {
        const double q = exp(logp);
        /* p = 1 - q < 0 has no normal quantile: the reference's cdfnor2 gives
           NaN there, and -inf (clamped to 0) at q == 1 */
        if (q > 1.0)
            return NAN;
        if (q == 1.0)
            return 0.0;
        x = norm_quantile_upper(q);
    }
    return x < 0.0 ? 0.0 : x;
}

double orc_candidate_sigma(double power, int numsum, double numtrials)
{
    double logp;
    if (power <= 0.0)
        return 0.0;
    logp = chi2_logp2(2.0 * power, 2.0 * numsum);
    logp += log(numtrials);
    return equivalent_gaussian_sigma2(logp);
}

/* Summed power whose chi^2 tail (dof = 2*numsum), times numtrials, equals
 * the Gaussian tail at sigma.  Solved to full double precision by bisection
 * on log Q. */
double orc_power_for_sigma(double sigma, int numsum, double numtrials)
{
    double q = 0.5 * erfc(sigma / M_SQRT2) / numtrials;
    double logq = log(q);
    double lo = 0.0, hi = 1.0;
    while (log(q_gamma_int(numsum, hi)) > logq)
        hi *= 2.0;
    for (int it = 0; it < 200; it++) {
        double mid = 0.5 * (lo + hi);
        if (log(q_gamma_int(numsum, mid)) > logq)
            lo = mid;
        else
            hi = mid;
        if (hi - lo <= 1e-15 * hi)
            break;
    }
    return 0.5 * (lo + hi);
}

/* ------------------------------------------------------------------ */
/* Per-rstep volume                                                     */

/* Quickselect-free order statistic: the value of rank (n-1)/2, which is what
 * src/median.c returns (lower middle for even n). */
static int cmp_float(const void *a, const void *b)
{
    float fa = *(const float *)a, fb = *(const float *)b;
    return (fa > fb) - (fa < fb);
}

/* The reference's fast inverse square root (src/misc_utils.c:293-304): the
 * published bit-level first guess and one Newton step, in float.  The
 * reference is built with -ffast-math, and gcc then evaluates the Newton step
 * as y * (1.5 - (0.5 x)(y y)) -- bit-identical to the reference build over
 * 40,000 inputs, where the source order differs in about one case in six. */
static float invsqrtf_ref(float x)
{
    union {
        float f;
        int32_t i;
    } t;
    t.f = x;
    t.i = 0x5f3759df - (t.i >> 1);
    const float y = t.f;
    const float yy = y * y;
    const float hx = 0.5f * x;
    return y * (1.5f - hx * yy);
}

/* Local power levels of the -locpow normalisation (src/corr_routines.c:309-366,
 * used at src/accel_utils.c:1186-1203).  The reference correlates the powers,
 * through realfft / real_corr_conv (whose round trip scales by 2/n), with a
 * double top-hat of weight (n/2)/NUMLOCPOWAVG -- integer division -- at offsets
 * DELTAAVGBINS+1 .. NUMLOCPOWAVG/2+DELTAAVGBINS on both sides; restated as the
 * direct sum (checked against the reference's own routine to 2e-7).  The first
 * and last kern_half_width bins take the nearest interior value. */
#define LOC_NUMAVG 20 /* NUMLOCPOWAVG, include/presto.h:100 */
#define LOC_DELTA 5   /* DELTAAVGBINS, include/presto.h:104 */
static void local_powers(const float *p, int n, float *out)
{
    const int khw = LOC_NUMAVG / 2 + LOC_DELTA;
    const double w = (double)((n / 2) / LOC_NUMAVG) * 2.0 / (double)n;
    for (int i = khw; i < n - khw; i++) {
        double s = 0.0;
        for (int d = LOC_DELTA + 1; d <= khw; d++)
            s += (double)p[i + d] + (double)p[i - d];
        out[i] = (float)(w * s);
    }
    for (int i = 0; i < khw; i++) {
        out[i] = out[khw];
        out[n - 1 - i] = out[n - 1 - khw];
    }
}

static float median_of(float *arr, int n)
{
    qsort(arr, n, sizeof(float), cmp_float);
    return arr[(n - 1) / 2];
}

/* src/accel_utils.c:1058-1092: numbins complex values starting at lobin,
 * zero outside the file. */
static void get_amplitudes(const orc_geom *g, const float *fft, long long lobin, int numbins,
                           float *out)
{
    for (int ii = 0; ii < numbins; ii++) {
        long long b = lobin - g->lobin + ii;
        if (b < 0 || b >= g->numbins) {
            out[2 * ii] = 0.0f;
            out[2 * ii + 1] = 0.0f;
        } else {
            out[2 * ii] = fft[2 * b];
            out[2 * ii + 1] = fft[2 * b + 1];
        }
    }
}

typedef struct orc_vol {
    long long rlo;
    int zlo, wlo, numrs, numzs, numws;
    float *powers;            /* [numws][numzs][numrs] */
    unsigned short *rinds;    /* corr_uselen (subharmonics only) */
    unsigned short *zinds;    /* numz */
} orc_vol;

/* subharm_fderivs_vol, src/accel_utils.c:1094-1293 */
static int fderivs(const orc_geom *g, const orc_sub *s, const float *fft, double fullrlo,
                   double fullrhi, orc_vol *v)
{
    const int numharm = s->numharm, harmnum = s->harmnum;
    const double harm_fract = (double)harmnum / (double)numharm;
    const double drlo = calc_required_r(harm_fract, fullrlo);
    const double drhi = calc_required_r(harm_fract, fullrhi);
    const int fftlen = s->fftlen, binoffset = s->halfwidth;
    const int numdata = fftlen / ACCEL_NUMBETWEEN;
    float *data, *powers;
    double *pdata, *pfft, *tmp, *out;
    mixfft_plan *fwd, *inv;

    v->rlo = (long long)floor(drlo);
    v->zlo = calc_required_z(harm_fract, g->zlo);
    v->wlo = calc_required_w(harm_fract, g->wlo);
    v->rinds = NULL;
    v->zinds = NULL;
    if (numharm > 1) {
        v->rinds = (unsigned short *)malloc(sizeof(unsigned short) * g->corr_uselen);
        v->zinds = (unsigned short *)malloc(sizeof(unsigned short) * g->numz);
        for (int ii = 0; ii < g->corr_uselen; ii++) {
            double rr = fullrlo + ii * ACCEL_DR;
            double subr = calc_required_r(harm_fract, rr);
            v->rinds[ii] = (unsigned short)index_from_r(subr, (double)v->rlo);
        }
        for (int ii = 0; ii < g->numz; ii++) {
            double zz = g->zlo + ii * ACCEL_DZ;
            int subz = calc_required_z(harm_fract, zz);
            v->zinds[ii] = (unsigned short)index_from_z(subz, v->zlo);
        }
    }
    v->numrs = (int)((ceil(drhi) - floor(drlo)) * ACCEL_RDR + DBLCORRECT) + 1;
    if (numharm == 1 && harmnum == 1)
        v->numrs = g->corr_uselen;
    else if (v->numrs % ACCEL_RDR)
        v->numrs = (v->numrs / ACCEL_RDR + 1) * ACCEL_RDR;
    v->numzs = s->numz;
    v->numws = s->numw;

    /* data chunk, normalisation */
    data = (float *)malloc(sizeof(float) * 2 * numdata);
    get_amplitudes(g, fft, v->rlo - binoffset, numdata, data);
    if (g->nph > 0.0) {
        double norm = 1.0 / sqrt(g->nph);
        for (int ii = 0; ii < 2 * numdata; ii++)
            data[ii] *= norm;
    } else if (g->norm_type == 0) {
        double norm;
        powers = (float *)malloc(sizeof(float) * numdata);
        for (int ii = 0; ii < numdata; ii++) {
            float r = data[2 * ii], i = data[2 * ii + 1];
            float rr = r * r, ii2 = i * i; /* POWER() as two float products + sum */
            powers[ii] = rr + ii2;
        }
        norm = 1.0 / sqrt(median_of(powers, numdata) / log(2.0));
        free(powers);
        for (int ii = 0; ii < 2 * numdata; ii++)
            data[ii] *= norm;
    } else {
        /* -locpow: float norm per bin, invsqrtf of the local power */
        float *loc = (float *)malloc(sizeof(float) * numdata);
        powers = (float *)calloc((size_t)numdata, sizeof(float));
        for (int ii = 0; ii < numdata; ii++) {
            float r = data[2 * ii], i = data[2 * ii + 1];
            float rr = r * r, ii2 = i * i;
            powers[ii] = rr + ii2;
        }
        local_powers(powers, numdata, loc);
        for (int ii = 0; ii < numdata; ii++) {
            const float norm = invsqrtf_ref(loc[ii]);
            data[2 * ii] *= norm;
            data[2 * ii + 1] *= norm;
        }
        free(powers);
        free(loc);
    }

    /* spread_no_pad + forward FFT (double) */
    pdata = (double *)calloc(2 * (size_t)fftlen, sizeof(double));
    pfft = (double *)malloc(sizeof(double) * 2 * fftlen);
    for (int ii = 0; ii < numdata; ii++) {
        pdata[4 * ii] = data[2 * ii];
        pdata[4 * ii + 1] = data[2 * ii + 1];
    }
    free(data);
    fwd = mixfft_create(fftlen, -1);
    inv = mixfft_create(fftlen, +1);
    mixfft_exec(fwd, pdata, pfft);

    v->powers = (float *)malloc(sizeof(float) * (size_t)v->numws * v->numzs * v->numrs);
    tmp = (double *)malloc(sizeof(double) * 2 * fftlen);
    out = (double *)malloc(sizeof(double) * 2 * fftlen);
    {
        const double norm = 1.0 / ((double)fftlen * (double)fftlen);
        const int offset = binoffset * ACCEL_NUMBETWEEN;
        for (int ii = 0; ii < v->numws; ii++) {
            for (int jj = 0; jj < v->numzs; jj++) {
                const float *k = s->kern + 2L * ((long)ii * s->numz + jj) * fftlen;
                float *op = v->powers + ((long)ii * v->numzs + jj) * v->numrs;
                for (int kk = 0; kk < fftlen; kk++) {
                    const double dr = pfft[2 * kk], di = pfft[2 * kk + 1];
                    const double kr = k[2 * kk], ki = k[2 * kk + 1];
                    tmp[2 * kk] = dr * kr + di * ki;
                    tmp[2 * kk + 1] = di * kr - dr * ki;
                }
                mixfft_exec(inv, tmp, out);
                for (int kk = 0; kk < v->numrs; kk++) {
                    const int ind = 2 * (kk + offset);
                    op[kk] = (float)((out[ind] * out[ind] + out[ind + 1] * out[ind + 1]) * norm);
                }
            }
        }
    }
    free(tmp);
    free(out);
    free(pdata);
    free(pfft);
    mixfft_destroy(fwd);
    mixfft_destroy(inv);
    return 0;
}

static void free_vol(orc_vol *v)
{
    free(v->powers);
    free(v->rinds);
    free(v->zinds);
}

/* add_ffdotpows, src/accel_utils.c:1356-1377 */
static void add_vol(orc_vol *fund, const orc_vol *sub, int numharm, int harmnum)
{
    const double harm_fract = (double)harmnum / (double)numharm;
    for (int ii = 0; ii < fund->numws; ii++) {
        int ww = fund->wlo + ii * ACCEL_DW;
        int subw = calc_required_w(harm_fract, ww);
        int wind = index_from_w(subw, sub->wlo);
        for (int jj = 0; jj < fund->numzs; jj++) {
            int zind = sub->zinds[jj];
            const float *in = sub->powers + ((long)wind * sub->numzs + zind) * sub->numrs;
            float *o = fund->powers + ((long)ii * fund->numzs + jj) * fund->numrs;
            for (int kk = 0; kk < fund->numrs; kk++)
                o[kk] += in[sub->rinds[kk]];
        }
    }
}

/* ------------------------------------------------------------------ */
/* Candidate list: insert_new_accelcand, src/accel_utils.c:382-480.       */
/* The list is an array in list order; the walk is the reference's linear   */
/* walk ("first node with r >= rr, else the last node").  The list is NOT   */
/* always sorted: when the walk ends at the last node (r < rr) and only the */
/* node before it is overwritten, the new r lands before a smaller one.     */

typedef struct cand_list {
    orc_cand *c;
    long n, cap;
} cand_list;

static void list_insert_at(cand_list *L, long pos, orc_cand v)
{
    if (L->n == L->cap) {
        L->cap = L->cap ? 2 * L->cap : 1024;
        L->c = (orc_cand *)realloc(L->c, sizeof(orc_cand) * L->cap);
    }
    memmove(L->c + pos + 1, L->c + pos, sizeof(orc_cand) * (L->n - pos));
    L->c[pos] = v;
    L->n++;
}

static void list_remove_at(cand_list *L, long pos)
{
    memmove(L->c + pos, L->c + pos + 1, sizeof(orc_cand) * (L->n - pos - 1));
    L->n--;
}

static int insert_cand(cand_list *L, orc_cand v)
{
    long tmp, prev;
    double prev_diff_r = ACCEL_CLOSEST_R + 1.0, next_diff_r;
    int added = 0;
    if (L->n == 0) {
        list_insert_at(L, 0, v);
        return 1;
    }
    tmp = 0;
    while (tmp < L->n - 1 && L->c[tmp].r < v.r)
        tmp++;
    prev = tmp - 1;
    next_diff_r = fabs(v.r - L->c[tmp].r);
    if (prev >= 0)
        prev_diff_r = fabs(v.r - L->c[prev].r);
    if (prev_diff_r < ACCEL_CLOSEST_R) {
        if (L->c[prev].sigma < v.sigma) {
            L->c[prev] = v;
            added = 1;
        }
        if (next_diff_r < ACCEL_CLOSEST_R) {
            if (L->c[tmp].sigma < v.sigma) {
                if (added) {
                    list_remove_at(L, tmp);
                } else {
                    L->c[tmp] = v;
                    added = 1;
                }
            }
        }
    } else if (next_diff_r < ACCEL_CLOSEST_R) {
        if (L->c[tmp].sigma < v.sigma) {
            L->c[tmp] = v;
            added = 1;
        }
    } else {
        added = 1;
        if (tmp == L->n - 1 && L->c[tmp].r < v.r - ACCEL_CLOSEST_R)
            list_insert_at(L, tmp + 1, v);
        else
            list_insert_at(L, tmp, v);
    }
    return added;
}

/* Optional record of every threshold crossing, keyed like the product's
 * hits: ((((rstep * numharmstages + stage) * numw + ii) * numz + jj) * numrs + kk */
typedef struct hit_rec {
    unsigned long long *keys;
    float *pows;
    long n, cap;
    long long rstep;
} hit_rec;

static void rec_hit(hit_rec *h, const orc_geom *g, const orc_vol *f, int stage, int ii, int jj,
                    int kk, float pw)
{
    if (!h)
        return;
    if (h->n < h->cap) {
        h->keys[h->n] = ((((unsigned long long)h->rstep * g->numharmstages + stage) * f->numws +
                          ii) * f->numzs + jj) * f->numrs + kk;
        h->pows[h->n] = pw;
    }
    h->n++;
}

/* search_ffdotpows, src/accel_utils.c:1507-1555 (single thread order) */
static void search_vol(const orc_geom *g, const orc_vol *f, int numharm, cand_list *L,
                       long *nhits, hit_rec *hr)
{
    int stage = 0;
    while ((1 << stage) < numharm)
        stage++;
    const float powcut = g->powcut[stage];
    const long long numindep = g->numindep[stage];
    for (int ii = 0; ii < f->numws; ii++)
        for (int jj = 0; jj < f->numzs; jj++)
            for (int kk = 0; kk < f->numrs; kk++) {
                float pw = f->powers[((long)ii * f->numzs + jj) * f->numrs + kk];
                if (pw > powcut) {
                    orc_cand c;
                    c.power = pw;
                    c.sigma = (float)orc_candidate_sigma(pw, numharm, (double)numindep);
                    c.numharm = numharm;
                    c.r = (f->rlo + kk * (double)ACCEL_DR) / (double)numharm;
                    c.z = (f->zlo + jj * (double)ACCEL_DZ) / (double)numharm;
                    c.w = (f->wlo + ii * (double)ACCEL_DW) / (double)numharm;
                    insert_cand(L, c);
                    rec_hit(hr, g, f, stage, ii, jj, kk, pw);
                    (*nhits)++;
                }
            }
}

/* ------------------------------------------------------------------ */
/* Exported entry points                                                */

/* One subharmonic volume.  hdr: rlo, zlo, wlo, numrs, numzs, numws.
 * powers/rinds/zinds may be NULL (then only hdr is filled). */
int orc_fderivs(const orc_geom *g, const orc_sub *s, const float *fft, double fullrlo,
                double fullrhi, long long *hdr, float *powers, unsigned short *rinds,
                unsigned short *zinds)
{
    orc_vol v;
    fderivs(g, s, fft, fullrlo, fullrhi, &v);
    hdr[0] = v.rlo;
    hdr[1] = v.zlo;
    hdr[2] = v.wlo;
    hdr[3] = v.numrs;
    hdr[4] = v.numzs;
    hdr[5] = v.numws;
    if (powers)
        memcpy(powers, v.powers, sizeof(float) * (size_t)v.numws * v.numzs * v.numrs);
    if (rinds && v.rinds)
        memcpy(rinds, v.rinds, sizeof(unsigned short) * g->corr_uselen);
    if (zinds && v.zinds)
        memcpy(zinds, v.zinds, sizeof(unsigned short) * g->numz);
    free_vol(&v);
    return 0;
}

/* The fundamental of one rstep after harmonic summing through 'stage'
 * (powers [numw][numz][corr_uselen]). */
int orc_summed(const orc_geom *g, const orc_sub *subs, const float *fft, double startr,
               int upto_stage, float *powers)
{
    orc_vol fund;
    const double lastr = startr + g->corr_uselen * ACCEL_DR - ACCEL_DR;
    int idx = 1;
    fderivs(g, &subs[0], fft, startr, lastr, &fund);
    for (int stage = 1; stage <= upto_stage && stage < g->numharmstages; stage++) {
        int harmtosum = 1 << stage;
        for (int harm = 1; harm < harmtosum; harm += 2, idx++) {
            orc_vol sub;
            fderivs(g, &subs[idx], fft, startr, lastr, &sub);
            add_vol(&fund, &sub, harmtosum, harm);
            free_vol(&sub);
        }
    }
    memcpy(powers, fund.powers, sizeof(float) * (size_t)fund.numws * fund.numzs * fund.numrs);
    free_vol(&fund);
    return 0;
}

/* The accelsearch loop (src/accelsearch.c:183-223) from rstep 'first_step'
 * for at most max_steps rsteps (all when <= 0).  subs are in bank order:
 * (1/1), (1/2), (1/4), (3/4), (1/8), ...  Returns the number of candidates
 * in the final list; up to max_out are copied to out.  *nhits receives the
 * number of threshold crossings (every call to insert). */
long orc_search_hits(const orc_geom *g, const orc_sub *subs, const float *fft, long first_step,
                     long max_steps, orc_cand *out, long max_out, long *steps_done, long *nhits,
                     unsigned long long *hit_keys, float *hit_pows, long hit_cap)
{
    cand_list L = {NULL, 0, 0};
    hit_rec hr = {hit_keys, hit_pows, 0, hit_keys ? hit_cap : 0, 0};
    hit_rec *hp = hit_keys ? &hr : NULL;
    const int rstep = g->corr_uselen * ACCEL_DR;
    double startr = g->rlo + (double)first_step * rstep;
    long nsteps = 0, n;
    *nhits = 0;
    while (startr + rstep < g->highestbin && (max_steps <= 0 || nsteps < max_steps)) {
        const double nextr = startr + rstep;
        const double lastr = nextr - ACCEL_DR;
        orc_vol fund;
        int idx = 1;
        hr.rstep = first_step + nsteps;
        fderivs(g, &subs[0], fft, startr, lastr, &fund);
        search_vol(g, &fund, 1, &L, nhits, hp);
        for (int stage = 1; stage < g->numharmstages; stage++) {
            int harmtosum = 1 << stage;
            for (int harm = 1; harm < harmtosum; harm += 2, idx++) {
                orc_vol sub;
                fderivs(g, &subs[idx], fft, startr, lastr, &sub);
                add_vol(&fund, &sub, harmtosum, harm);
                free_vol(&sub);
            }
            search_vol(g, &fund, harmtosum, &L, nhits, hp);
        }
        free_vol(&fund);
        startr = nextr;
        nsteps++;
    }
    n = L.n;
    if (out)
        memcpy(out, L.c, sizeof(orc_cand) * (size_t)(n < max_out ? n : max_out));
    free(L.c);
    if (steps_done)
        *steps_done = nsteps;
    return n;
}

long orc_search(const orc_geom *g, const orc_sub *subs, const float *fft, long first_step,
                long max_steps, orc_cand *out, long max_out, long *steps_done, long *nhits)
{
    return orc_search_hits(g, subs, fft, first_step, max_steps, out, max_out, steps_done, nhits,
                           NULL, NULL, 0);
}

/* Apply insert_new_accelcand to a given hit sequence (power, numharm, r, z,
 * w already decoded, sigma computed here); returns the final list. */
long orc_insert_hits(const orc_cand *hits, long nhits, const long long *numindep,
                     orc_cand *out, long max_out)
{
    cand_list L = {NULL, 0, 0};
    long n;
    for (long i = 0; i < nhits; i++) {
        orc_cand c = hits[i];
        int stage = 0;
        while ((1 << stage) < c.numharm)
            stage++;
        c.sigma = (float)orc_candidate_sigma(c.power, c.numharm, (double)numindep[stage]);
        insert_cand(&L, c);
    }
    n = L.n;
    if (out)
        memcpy(out, L.c, sizeof(orc_cand) * (size_t)(n < max_out ? n : max_out));
    free(L.c);
    return n;
}

/* exported for pinning against the reference build */
void orc_local_powers(const float *p, int n, float *out) { local_powers(p, n, out); }
float orc_invsqrtf(float x) { return invsqrtf_ref(x); }

/* ------------------------------------------------------------------ */
/* Red-noise removal of a spectrum read from a time series              */

/* deredden (src/accel_utils.c:1557-1633): the powers are split into blocks
 * that start at bin 1 with 6 bins and grow as 6 ln(start bin) (at most 200),
 * while a whole block still fits below numamps.  Each block's level is its
 * median power (rank (n-1)/2, src/median.c) over ln 2.  Bins are scaled by
 * invsqrtf of a level that runs linearly from one block's level to the
 * next's, across the second half of one block and the first half of the
 * next; the first half block takes the first level and the tail past the
 * last block extends the last slope.  The DC bin becomes (1, 0).  All
 * arithmetic in the reference's types: powers and levels in float, the
 * division by ln 2 and by the half block sum in double. */
void orc_deredden(float *fft, int numamps)
{
    const int initlen = 6, maxlen = 200;
    float *pw = malloc(sizeof(float) * (size_t)numamps), *tmp = malloc(sizeof(float) * maxlen);
    fft[0] = 1.0f;
    fft[1] = 0.0f;
    for (int i = 0; i < numamps; i++)
        pw[i] = fft[2 * i] * fft[2 * i] + fft[2 * i + 1] * fft[2 * i + 1];
    int binnum = 1, numwrote = 1, buflen = initlen, lastlen;
    memcpy(tmp, pw + binnum, sizeof(float) * buflen);
    float mean_old = (float)(median_of(tmp, buflen) / log(2.0)), dslope = 1.0f;
    const float norm0 = invsqrtf_ref(mean_old);
    for (int k = numwrote; k < binnum + buflen / 2; k++) {
        fft[2 * k] *= norm0;
        fft[2 * k + 1] *= norm0;
    }
    numwrote += buflen / 2;
    binnum += buflen;
    lastlen = buflen;
    buflen = (int)(initlen * log((double)binnum));
    if (buflen > maxlen)
        buflen = maxlen;
    while (binnum + buflen < numamps) {
        memcpy(tmp, pw + binnum, sizeof(float) * buflen);
        const float mean_new = (float)(median_of(tmp, buflen) / log(2.0));
        dslope = (float)((double)(mean_new - mean_old) / (0.5 * (double)(lastlen + buflen)));
        int ii = 0;
        for (int k = numwrote; k < binnum + buflen / 2; k++, ii++) {
            const float norm = invsqrtf_ref(mean_old + dslope * (float)ii);
            fft[2 * k] *= norm;
            fft[2 * k + 1] *= norm;
        }
        numwrote += ii;
        binnum += buflen;
        lastlen = buflen;
        mean_old = mean_new;
        buflen = (int)(initlen * log((double)binnum));
        if (buflen > maxlen)
            buflen = maxlen;
    }
    for (int k = numwrote, ii = 0; k < numamps; k++, ii++) {
        const float norm = invsqrtf_ref(mean_old + dslope * (float)ii);
        fft[2 * k] *= norm;
        fft[2 * k + 1] *= norm;
    }
    free(pw);
    free(tmp);
}

/* ------------------------------------------------------------------ */
/* Birdie zapping of a spectrum held in memory                          */

#define ZAP_MEDIANBINS 200 /* MEDIANBINS, src/zapping.c:3 */

/* Median power (rank (n-1)/2) of n bins from fft + first; bins at or past
 * numamps read as zeros (the reference's .dat buffer is zero-padded there,
 * ACCEL_PADDING, include/accel.h:35). */
static float zap_median(const float *fft, long numamps, long first, int n)
{
    float *p = malloc(sizeof(float) * (size_t)n);
    for (int i = 0; i < n; i++) {
        const long b = first + i;
        const float r = (b >= 0 && b < numamps) ? fft[2 * b] : 0.0f;
        const float im = (b >= 0 && b < numamps) ? fft[2 * b + 1] : 0.0f;
        p[i] = r * r + im * im;
    }
    const float m = median_of(p, n);
    free(p);
    return m;
}

/* zapbirds from memory (src/zapping.c:29-81): when the birdie starts above
 * 1.5 MEDIANBINS + 1, the bins [floor(lobin), ceil(hibin)) take the amplitude
 * sqrt(mean of the median powers below and above it / ln 2), phase 0. */
void orc_zapbirds(float *fft, long numamps, double lobin, double hibin)
{
    const long ilobin = (long)floor(lobin), ihibin = (long)ceil(hibin);
    if (!(lobin - 1.5 * ZAP_MEDIANBINS > 1))
        return;
    const float mlo = zap_median(fft, numamps, (long)(lobin - 3 * ZAP_MEDIANBINS / 2),
                                 ZAP_MEDIANBINS);
    const float mhi = zap_median(fft, numamps, (long)(hibin - ZAP_MEDIANBINS / 2),
                                 ZAP_MEDIANBINS);
    const float avgamp = (float)sqrt(0.5 * (mlo + mhi) / -log(0.5));
    for (long b = ilobin; b < ihibin; b++) {
        fft[2 * b] = avgamp;
        fft[2 * b + 1] = 0.0f;
    }
}

/* The caller's loop (src/accelsearch_lib.c:393-418): birdies in list order,
 * stopping at the first one at or above N/2 bins, high edges clamped to
 * N/2 - 1. */
void orc_zap_list(float *fft, long numamps, long long N, const double *lobins,
                  const double *hibins, int nbirds)
{
    const double top = (double)(N / 2);
    for (int i = 0; i < nbirds; i++) {
        if (lobins[i] >= top)
            break;
        orc_zapbirds(fft, numamps, lobins[i], hibins[i] >= top ? top - 1 : hibins[i]);
    }
}

/* Subband downsampling (prepsubband's get_data, src/prepsubband.c:984-1001;
 * on the GPU DownsampDataArray, src/prepsubband_kernels.cu:23-46): blocks of
 * worklen output samples of nsub subbands, time-major; each output the FP32
 * sum of bs consecutive inputs of its subband, in time order, divided by bs. */
void orc_downsample_subbands(float *out, const float *in, int worklen, int bs, int nsub)
{
    for (long t = 0; t < worklen; t++)
        for (int s = 0; s < nsub; s++) {
            float acc = 0.0f;
            for (int k = 0; k < bs; k++)
                acc += in[((long)t * bs + k) * nsub + s];
            out[t * nsub + s] = acc / (float)bs;
        }
}

/* Subband dedispersion (float_dedisp with approx_mean 0, src/dispersion.c:
 * 208-231, as prepsubband calls it per DM, src/prepsubband.c:1010-1013): for
 * DM d, out[d][t] starts at -0.0f and adds, subband by subband in ascending
 * order, sample t + offsets[d][s] of the previous block (last) followed by
 * the current one (cur). */
void orc_dedisp_subbands(const float *cur, const float *last, float *out, int worklen, int nsub,
                         int numdms, const int *offsets)
{
    for (int d = 0; d < numdms; d++) {
        float *row = out + (long)d * worklen;
        for (long t = 0; t < worklen; t++)
            row[t] = -0.0f;
        for (int s = 0; s < nsub; s++) {
            const long off = offsets[(long)d * nsub + s];
            for (long t = 0; t < worklen; t++) {
                const long tau = t + off;
                row[t] += tau < worklen ? last[tau * nsub + s] : cur[(tau - worklen) * nsub + s];
            }
        }
    }
}
