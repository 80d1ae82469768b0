/*
 * Stand-in for the subset of the FFTW 3 single-precision API that the
 * reference PRESTO sources call (fftcalls.c, vectors.c, accel_utils.c,
 * fastffts.c).  FFTW itself is not installed in this image, so the oracle's
 * reference build links against this header and oracle/shim/fftw_shim.c
 * instead.
 *
 * TEST INFRASTRUCTURE ONLY: nothing in the product library includes this.
 *
 * Conventions follow FFTW's published documentation: sign -1 is the forward
 * transform exp(-2*pi*i*j*k/n), sign +1 the backward one, both unnormalised.
 * The transforms are computed in double precision internally and rounded to
 * float on output, so they are at least as accurate as FFTW's float path;
 * results therefore differ from a real-FFTW run only by float rounding.
 */
#ifndef ORACLE_SHIM_FFTW3_H
#define ORACLE_SHIM_FFTW3_H

#include <stdio.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef float fftwf_complex[2];
typedef struct fftwf_plan_s *fftwf_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)

#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_UNALIGNED (1U << 1)
#define FFTW_CONSERVE_MEMORY (1U << 2)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_WISDOM_ONLY (1U << 21)

fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out,
                             int sign, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_execute_dft(const fftwf_plan p, fftwf_complex *in, fftwf_complex *out);
void fftwf_destroy_plan(fftwf_plan p);
void *fftwf_malloc(size_t n);
void fftwf_free(void *p);
int fftwf_import_system_wisdom(void);
int fftwf_import_wisdom_from_file(FILE *input_file);
int fftwf_import_wisdom_from_filename(const char *filename);
void fftwf_export_wisdom_to_file(FILE *output_file);
int fftwf_export_wisdom_to_filename(const char *filename);
void fftwf_forget_wisdom(void);
void fftwf_cleanup(void);

#ifdef __cplusplus
}
#endif

#endif
