/*
 * Link-time stand-ins for FFTW and PRESTO routines that the reference
 * libpresto objects reference but that the accelsearch path never calls
 * (tablesixstepfft's out-of-core transposes and its many-transform plans).
 * Each aborts loudly if it is ever reached, so a silent wrong answer is
 * impossible.
 *
 * TEST INFRASTRUCTURE ONLY.
 */
#include <stdio.h>
#include <stdlib.h>

#include "fftw3.h"

static void unreachable(const char *name)
{
    fprintf(stderr, "oracle shim: %s is not available in the oracle build\n", name);
    abort();
}

fftwf_plan fftwf_plan_many_dft(int rank, const int *n, int howmany, fftwf_complex *in,
                               const int *inembed, int istride, int idist,
                               fftwf_complex *out, const int *onembed, int ostride,
                               int odist, int sign, unsigned flags)
{
    (void)rank; (void)n; (void)howmany; (void)in; (void)inembed; (void)istride;
    (void)idist; (void)out; (void)onembed; (void)ostride; (void)odist; (void)sign;
    (void)flags;
    unreachable("fftwf_plan_many_dft");
    return NULL;
}

int transpose_fcomplex(void *a, int nx, int ny, unsigned char *move, int move_size)
{
    (void)a; (void)nx; (void)ny; (void)move; (void)move_size;
    unreachable("transpose_fcomplex");
    return 0;
}

/* src/dispersion.c (linked for float_dedisp) refers to these two from
 * subband_delays and combine_subbands, which the oracle never calls. */
double doppler(double freq_observed, double voverc)
{
    (void)freq_observed; (void)voverc;
    unreachable("doppler");
    return 0.0;
}

void initialize_foldstats(void *stats)
{
    (void)stats;
    unreachable("initialize_foldstats");
}
