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
 * first call and made again whenever the sizes or the table change
 * (prepsubband_cu uploads the table once per run).  Like the reference's
 * CUDA_CHECK, a failure prints the error and exits.
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

void getDedisp(float *currentdsdata_gpu, float *lastdsdata_gpu, float *outdata_gpu, int worklen,
               int nsub, int numdms, int *offsets)
{
    if (!g_dedisp || !jerk_dedisperser_matches(g_dedisp, worklen, nsub, numdms, offsets)) {
        jerk_dedisperser_destroy(g_dedisp);
        g_dedisp = NULL;
        if (jerk_dedisperser_create(&g_dedisp, worklen, nsub, numdms, offsets) != JERK_OK) {
            fprintf(stderr, "getDedisp: %s\n", jerk_last_error());
            exit(1);
        }
    }
    if (jerk_dedisp_subbands(g_dedisp, currentdsdata_gpu, lastdsdata_gpu, outdata_gpu, NULL) !=
        JERK_OK) {
        fprintf(stderr, "getDedisp: %s\n", jerk_last_error());
        exit(1);
    }
}
