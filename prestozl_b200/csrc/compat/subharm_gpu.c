/*
 * create_subharminfos without the kernels: the drop-in's half of moving the
 * kernel bank to the GPU.
 *
 * Same symbol, argument and result type as the reference's
 *     subharminfo **create_subharminfos(accelobs *obs)
 * (src/accel_utils.c:236-282), which accelsearch_CPU1 calls
 * (src/accelsearch_lib.c:423).  The drop-in build compiles the reference's
 * accel_utils.c with that function renamed to reference_create_subharminfos.
 *
 * The reference computes every response kernel of the bank here, on the
 * host: 2.9 s on one core for the paper configuration (-zmax 200 -wmax 300
 * -numharm 16).  The drop-in's accelsearch_GPU (compat/accelsearch_gpu.c)
 * uploads no kernels: it generates the bank on the GPU (jerk_bank_generate)
 * whenever the kernels' data pointers are NULL.  So this builds the same
 * structures -- the subharmonic geometry, the (z, w) kernel grid with each
 * kernel's z, w, fftlen, numbetween, kern_half_width and numgoodbins, the
 * rinds/zinds tables the reference allocates -- with data left NULL.
 * free_subharminfos (src/accel_utils.c:303-325) frees them unchanged.
 *
 * The geometry comes from jerk_subharm_sizes, this project's restatement of
 * the reference's sizing (init_subharminfo, calc_fftlen), which the tests
 * pin against the reference's own values.  In-memory searches (-inmem), which
 * the GPU search does not take, get the reference's routine.
 */
#include <stdio.h>
#include <stdlib.h>

#include "accel.h"
#include "jerk.h"
#include "jerk_compat.h"

subharminfo **reference_create_subharminfos(accelobs *obs);
kernel **gen_kernmatrix(int numz, int numw); /* src/accel_utils.c:170-192 */

static void fill_subharminfo(const jerk_subharm *sub, const accelobs *obs, subharminfo *shi)
{
    shi->numharm = sub->numharm;
    shi->harmnum = sub->harmnum;
    shi->zmax = sub->zmax;
    shi->wmax = sub->wmax;
    shi->rinds = NULL;
    shi->zinds = NULL;
    if (sub->numharm > 1) {
        shi->rinds = (unsigned short *)malloc(obs->corr_uselen * sizeof(unsigned short));
        shi->zinds = (unsigned short *)malloc(obs->corr_uselen * sizeof(unsigned short));
    }
    shi->numkern_zdim = sub->numz;
    shi->numkern_wdim = sub->numw;
    shi->numkern = sub->numz * sub->numw;
    shi->kern = gen_kernmatrix(sub->numz, sub->numw);
    for (int ii = 0; ii < sub->numw; ii++)
        for (int jj = 0; jj < sub->numz; jj++) {
            kernel *k = &shi->kern[ii][jj];
            k->z = -sub->zmax + jj * ACCEL_DZ;
            k->w = -sub->wmax + ii * ACCEL_DW;
            k->fftlen = sub->fftlen;
            k->numbetween = ACCEL_NUMBETWEEN;
            k->kern_half_width = w_resp_halfwidth((double)k->z, (double)k->w, LOWACC);
            k->numgoodbins = k->fftlen - 2 * k->numbetween * k->kern_half_width;
            k->data = NULL;
        }
}

subharminfo **create_subharminfos(accelobs *obs)
{
    if (obs->inmem)
        return reference_create_subharminfos(obs);
    jerk_obs o;
    jerk_obs_of_accelobs(obs, &o);
    const int nsubs = jerk_subharm_count(obs->numharmstages);
    jerk_subharm *subs = (jerk_subharm *)calloc(nsubs, sizeof(jerk_subharm));
    for (int i = 0; i < nsubs; i++)
        if (jerk_subharm_sizes(&o, obs->fftlen, i, &subs[i]) != JERK_OK) {
            fprintf(stderr, "create_subharminfos: %s\n", jerk_last_error());
            free(subs);
            return reference_create_subharminfos(obs);
        }
    /* layout of src/accel_utils.c:236-282: shis[0][0] the fundamental, then
       shis[stage][harm - 1] for the odd harms of 2^stage, in bank order */
    subharminfo **shis = (subharminfo **)malloc(obs->numharmstages * sizeof(subharminfo *));
    shis[0] = (subharminfo *)malloc(2 * sizeof(subharminfo));
    fill_subharminfo(&subs[0], obs, &shis[0][0]);
    int idx = 1;
    for (int ii = 1; ii < obs->numharmstages; ii++) {
        const int harmtosum = 1 << ii;
        shis[ii] = (subharminfo *)malloc(harmtosum * sizeof(subharminfo));
        for (int jj = 1; jj < harmtosum; jj += 2, idx++)
            fill_subharminfo(&subs[idx], obs, &shis[ii][jj - 1]);
    }
    free(subs);
    return shis;
}
