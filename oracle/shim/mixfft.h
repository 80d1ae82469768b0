/*
 * Double-precision mixed-radix complex FFT used by the oracle: by the FFTW
 * stand-in (fftw_shim.c) that the reference build links, and directly by the
 * oracle's own restatement of the search (oracle/jerk_oracle.c).
 *
 * TEST INFRASTRUCTURE ONLY.
 *
 * Algorithm: textbook recursive Cooley-Tukey decimation in time over the
 * factors of n (radix 4, 2, 3, 5, then any remaining prime by a direct DFT),
 * with one exp(sign*2*pi*i*k/n) table per plan.  Unnormalised, sign -1 is the
 * forward transform.
 */
#ifndef ORACLE_MIXFFT_H
#define ORACLE_MIXFFT_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mixfft_plan mixfft_plan;

/* Plan a length-n transform with exponent sign 'sign' (-1 or +1). */
mixfft_plan *mixfft_create(int n, int sign);
void mixfft_destroy(mixfft_plan *p);
int mixfft_size(const mixfft_plan *p);

/* out[k] = sum_j in[j] * exp(sign*2*pi*i*j*k/n); interleaved (re, im)
 * doubles; in and out must not overlap.  Thread-safe for one plan. */
void mixfft_exec(const mixfft_plan *p, const double *in, double *out);

#ifdef __cplusplus
}
#endif

#endif
