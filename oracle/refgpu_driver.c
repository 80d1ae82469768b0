/*
 * Timing driver for the REFERENCE's own GPU search stage (TEST AND BENCH
 * INFRASTRUCTURE ONLY).
 *
 * Runs the reference's three stages on one .fft file exactly as its
 * accelsearch_cu CLI does (src/accelsearch_cu.c:22-34: accelsearch_CPU1, then
 * accelsearch_GPU, then accelsearch_CPU2 from src/accelsearch_lib.c), and
 * prints the wall time of the GPU stage -- the reference's plain search loop:
 * kernel-bank upload, per-rstep host preparation, cuFFT correlation, fused
 * harmonic sum and candidate insertion -- as one JSON line on stderr.  The
 * bank generation (inside CPU1) and the ACCEL writing (CPU2) are outside the
 * timed region, as they are outside libjerk's search too.
 */
#include <stdio.h>
#include <sys/time.h>

#include "accel.h"

static double now_s(void)
{
    struct timeval tv;
    gettimeofday(&tv, NULL);
    return (double)tv.tv_sec + 1e-6 * (double)tv.tv_usec;
}

int main(int argc, char *argv[])
{
    subharminfo **subs = NULL;
    accelobs obs;
    infodata idata;
    GSList *cands = NULL;
    Cmdline *cmd = NULL;

    accelsearch_CPU1(argc, argv, &subs, &obs, &idata, &cmd);
    const double t0 = now_s();
    const int rc = accelsearch_GPU(obs, subs, &cands, cmd);
    const double t1 = now_s();
    const unsigned ncands = g_slist_length(cands);
    accelsearch_CPU2(&cands, &obs, &idata, cmd);
    fprintf(stderr, "{\"refgpu_search_s\": %.6f, \"rc\": %d, \"ncands\": %u}\n", t1 - t0, rc,
            ncands);
    return rc;
}
