/*
 * The GPU steps of prepsubband_cu over libjerk: the drop-in for the
 * reference's src/prepsubband_kernels.cu.
 *
 * Same symbols, arguments and results as the reference's
 *     void DownsampDataArray(float *currentdsdata_gpu, float *currentdata_gpu,
 *                            int worklen, int bs, int nsub)
 *     void getDedisp(float *currentdsdata_gpu, float *lastdsdata_gpu,
 *                    float *outdata_gpu, int worklen, int nsub, int numdms,
 *                    int *offsets)
 * (src/prepsubband_kernels.cu:21-22, 76-87), which prepsubband_cu calls
 * per block of subband data (src/prepsubband_cu.c:1140-1165) on device
 * buffers.  Linking this file in place of prepsubband_kernels.cu gives the
 * same DM-trial series bit for bit (tests/test_gpu_dedisp.py).
 *
 * Both run on the legacy default stream, as the reference's launches do, so
 * the reference's synchronous cudaMemcpy calls around them order as before.
 * getDedisp keeps one jerk_dedisperser, made from the offsets table on its
 * first call.  prepsubband_cu uploads the table to one device buffer once per
 * run, before its block loop (src/prepsubband_cu.c:380, 481-488, 611-618), so
 * a call with the same table pointer and sizes reuses the dedisperser with
 * no check; a new pointer or new sizes compare the table
 * (jerk_dedisperser_matches, one device-to-host copy of numdms * nsub ints)
 * and make a new dedisperser if it differs.  A caller that rewrites the table
 * in place between blocks must free it and upload to a new buffer, or the
 * old offsets stay in use.  Like the reference's CUDA_CHECK, a failure prints
 * the error and exits.
 */
#include <stdio.h>
#include <stdlib.h>

#include "jerk.h"

void DownsampDataArray(float *currentdsdata_gpu, float *currentdata_gpu, int worklen, int bs,
                       int nsub)
{
    if (jerk_downsample_subbands(currentdsdata_gpu, currentdata_gpu, worklen, bs, nsub, NULL) !=
        JERK_OK) {
        fprintf(stderr, "DownsampDataArray: %s\n", jerk_last_error());
        exit(1);
    }
}

static jerk_dedisperser *g_dedisp;
static const int *g_offsets;  /* the table pointer and sizes g_dedisp was last used with */
static int g_worklen, g_nsub, g_numdms;

void getDedisp(float *currentdsdata_gpu, float *lastdsdata_gpu, float *outdata_gpu, int worklen,
               int nsub, int numdms, int *offsets)
{
    const int same_call = g_dedisp && offsets == g_offsets && worklen == g_worklen &&
                          nsub == g_nsub && numdms == g_numdms;
    if (!same_call && (!g_dedisp ||
                       !jerk_dedisperser_matches(g_dedisp, worklen, nsub, numdms, offsets))) {
        jerk_dedisperser_destroy(g_dedisp);
        g_dedisp = NULL;
        if (jerk_dedisperser_create(&g_dedisp, worklen, nsub, numdms, offsets) != JERK_OK) {
            fprintf(stderr, "getDedisp: %s\n", jerk_last_error());
            exit(1);
        }
    }
    g_offsets = offsets;
    g_worklen = worklen;
    g_nsub = nsub;
    g_numdms = numdms;
    if (jerk_dedisp_subbands(g_dedisp, currentdsdata_gpu, lastdsdata_gpu, outdata_gpu, NULL) !=
        JERK_OK) {
        fprintf(stderr, "getDedisp: %s\n", jerk_last_error());
        exit(1);
    }
}
