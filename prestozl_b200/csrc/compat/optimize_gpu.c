/*
 * optimize_accelcand with the volume search on the GPU: the drop-in's
 * candidate optimisation for accelsearch_CPU2 (src/accelsearch_lib.c:903-975).
 *
 * Same symbol, arguments and results as the reference's
 *     void optimize_accelcand(accelcand *cand, accelobs *obs)
 * (src/accel_utils.c:573-657).  The drop-in build compiles the reference's
 * accel_utils.c with that function renamed to reference_optimize_accelcand,
 * so CPU2 calls this one.
 *
 * The reference's default path -- harmonic polishing of a search with -wmax
 * on a spectrum held in memory -- runs max_rzw_arr_harmonics
 * (src/maximize_rzw.c:84-190).  Here:
 *   - the local power of each harmonic (get_localpower3d) is the reference's
 *     own routine, as is everything after the volume search: the
 *     derivatives at the peak (get_derivs3d), the harmonic values and the
 *     sigma;
 *   - the volume search itself -- 17 x 17 response kernels per harmonic,
 *     their correlations and the summed-power maximum, about 98 % of the
 *     reference's optimisation time -- is jerk_polish_rzw on the GPU.
 * The polished (r, z, w) are grid points, equal to the reference's (see
 * tests/test_gpu_polish.py), so the ACCEL files are the reference's.
 *
 * The reference's other paths (no -wmax, -noharmpolish, spectra streamed
 * from the file) and candidates whose polishing FFTs exceed what the GPU
 * polisher takes (8192 points: about zmax 300 with wmax 600 and above) run
 * reference_optimize_accelcand unchanged.
 */
#include <stdio.h>
#include <stdlib.h>

#include "accel.h"
#include "jerk.h"

void reference_optimize_accelcand(accelcand *cand, accelobs *obs);

static jerk_polisher *g_polisher;
static int g_polisher_failed;

static int index_of_power_of_two(int n)
{
    int i = 0;
    while ((1 << i) < n)
        i++;
    return i;
}

void optimize_accelcand(accelcand *cand, accelobs *obs)
{
    const int nh = cand->numharm;
    if (!(obs->use_harmonic_polishing && (obs->mmap_file || obs->dat_input) && obs->numw) ||
        nh > 32) {
        reference_optimize_accelcand(cand, obs);
        return;
    }
    if (!g_polisher && !g_polisher_failed && jerk_polisher_create(&g_polisher, NULL) != JERK_OK) {
        fprintf(stderr, "optimize_accelcand: GPU polisher unavailable (%s)\n", jerk_last_error());
        g_polisher_failed = 1;
    }
    float locpow[32];
    const double rin = cand->r - obs->lobin, zin = cand->z, win = cand->w;
    for (int i = 0; i < nh; i++) {
        const int n = nh - i;
        locpow[i] = (float)get_localpower3d(obs->fft, obs->numbins, rin * n, zin * n, win * n);
    }
    double r, z, w;
    if (!g_polisher || jerk_polish_rzw(g_polisher, obs->fft, obs->numbins, nh, rin, zin, win,
                                       locpow, &r, &z, &w, NULL) != JERK_OK) {
        reference_optimize_accelcand(cand, obs);
        return;
    }
    cand->pows = gen_dvect(nh);
    cand->hirs = gen_dvect(nh);
    cand->hizs = gen_dvect(nh);
    cand->hiws = gen_dvect(nh);
    cand->derivs = (rderivs *)malloc(sizeof(rderivs) * nh);
    /* the derivatives at the peak (src/maximize_rzw.c:172-180) */
    for (int i = 0; i < nh; i++) {
        const int hh = i + 1;
        const double rr = r * hh, zz = z * hh, ww = w * hh;
        /* a float there, as the reference holds it */
        const float lp = (float)get_localpower3d(obs->fft, obs->numbins, rr, zz, ww);
        get_derivs3d(obs->fft, obs->numbins, rr, zz, ww, lp, &cand->derivs[i]);
        cand->pows[i] = cand->derivs[i].pow;
    }
    /* src/accel_utils.c:601-606, 655-656 */
    for (int i = 0; i < nh; i++) {
        cand->hirs[i] = (r + obs->lobin) * (i + 1);
        cand->hizs[i] = z * (i + 1);
        cand->hiws[i] = obs->numw ? w * (i + 1) : 0.0;
    }
    cand->sigma = candidate_sigma(cand->power, cand->numharm,
                                  obs->numindep[index_of_power_of_two(cand->numharm)]);
}
