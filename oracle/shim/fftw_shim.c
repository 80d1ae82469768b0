/*
 * FFTW 3 single-precision API subset over the oracle's double-precision
 * mixed-radix FFT (mixfft.c).  Linked only into the oracle's build of the
 * reference sources (oracle/_ref); never into the product library.
 *
 * TEST INFRASTRUCTURE ONLY.
 */
#include "fftw3.h"
#include "mixfft.h"

#include <stdlib.h>
#include <string.h>

struct fftwf_plan_s {
    mixfft_plan *fft;
    int n;
    fftwf_complex *in;
    fftwf_complex *out;
};

fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out,
                             int sign, unsigned flags)
{
    (void)flags;
    fftwf_plan p = (fftwf_plan)calloc(1, sizeof(*p));
    if (!p)
        return NULL;
    p->fft = mixfft_create(n, sign);
    if (!p->fft) {
        free(p);
        return NULL;
    }
    p->n = n;
    p->in = in;
    p->out = out;
    return p;
}

/* Per-thread double-precision scratch, grown as needed and kept for the
 * thread's life: no allocation per execute, and plans stay safe to execute
 * from several threads at once, as FFTW's new-array execute is. */
static __thread double *g_scratch;
static __thread size_t g_scratch_len;

void fftwf_execute_dft(const fftwf_plan p, fftwf_complex *in, fftwf_complex *out)
{
    const int n = p->n;
    const size_t need = 4 * (size_t)n;
    if (g_scratch_len < need) {
        double *grown = (double *)realloc(g_scratch, sizeof(double) * need);
        if (!grown)
            abort();
        g_scratch = grown;
        g_scratch_len = need;
    }
    double *a = g_scratch;
    double *b = a + 2 * (size_t)n;
    const float *fin = (const float *)in;
    float *fout = (float *)out;

    for (long k = 0; k < 2L * n; k++)
        a[k] = fin[k];
    mixfft_exec(p->fft, a, b);
    for (long k = 0; k < 2L * n; k++)
        fout[k] = (float)b[k];
}

void fftwf_execute(const fftwf_plan p) { fftwf_execute_dft(p, p->in, p->out); }

void fftwf_destroy_plan(fftwf_plan p)
{
    if (!p)
        return;
    mixfft_destroy(p->fft);
    free(p);
}

void *fftwf_malloc(size_t n)
{
    void *ptr = NULL;
    if (posix_memalign(&ptr, 64, n ? n : 1) != 0)
        return NULL;
    return ptr;
}

void fftwf_free(void *p) { free(p); }

/* Wisdom is a planning cache in FFTW; the stand-in plans nothing, so every
 * wisdom call succeeds and does nothing. */
int fftwf_import_system_wisdom(void) { return 1; }
int fftwf_import_wisdom_from_file(FILE *input_file)
{
    (void)input_file;
    return 1;
}
int fftwf_import_wisdom_from_filename(const char *filename)
{
    (void)filename;
    return 1;
}
void fftwf_export_wisdom_to_file(FILE *output_file) { (void)output_file; }
int fftwf_export_wisdom_to_filename(const char *filename)
{
    (void)filename;
    return 1;
}
void fftwf_forget_wisdom(void) {}
void fftwf_cleanup(void) {}
