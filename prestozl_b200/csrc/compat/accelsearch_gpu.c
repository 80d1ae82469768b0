/*
 * accelsearch_GPU on libjerk: the drop-in for PrestoZL's GPU search stage.
 *
 * Same symbol, arguments and ownership as the reference's
 *     int accelsearch_GPU(accelobs obs, subharminfo **subharminfs,
 *                         GSList **cands_ptr, Cmdline *cmd)
 * (src/accelsearch_lib.c:473-901, declared in include/accel.h:189), so the
 * reference's accelsearch_CPU1 / accelsearch_CPU2, its C main
 * (src/accelsearch_cu.c:22-34) and its ctypes process pool
 * (bin/accelsearch_pipeline_cu.py:278-280, 350-360) call it unchanged.
 *
 * This file is compiled against the reference's own headers (accel.h and
 * what it includes, glib among them) when libjerk is integrated into the
 * reference build; it is the only part of this project that sees those
 * types.  Everything below it is the plain C ABI of jerk.h.
 *
 * Semantics kept from the reference:
 *   - candidates arrive as the GSList the CPU search would build (the
 *     reference's insertion order and 15-bin rule), each accelcand allocated
 *     with malloc like create_accelcand (src/accel_utils.c:326-345);
 *   - subharminfs is freed here, as the reference frees it
 *     (src/accelsearch_lib.c:897);
 *   - the return value is 0 on success; on failure it is non-zero with
 *     *cands_ptr = NULL (the reference returns 1 on hit-buffer overflow,
 *     src/accelsearch_lib.c:748-782; here overflow is retried internally and
 *     only real errors return).
 * Deliberate difference: with -numharm 1 the reference's GPU path finds no
 * candidates (everything sits under numharmstages > 1,
 * src/accelsearch_lib.c:648); here stage 0 is searched, as the CPU search does.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "accel.h"
#include "jerk.h"
#include "jerk_compat.h"

/* The last GPU-generated kernel bank and the geometry it was made for.  A
 * process that searches many spectra of one geometry -- the reference's
 * worker pool (bin/accelsearch_pipeline_cu.py) calls accelsearch_GPU once per
 * .fft file -- generates it once; it stays on the device until the geometry
 * changes or the process exits. */
static void *g_bank;
static jerk_subharm *g_bank_subs;
static int g_bank_nsubs;

static int same_geometry(const jerk_subharm *a, const jerk_subharm *b, int n)
{
    for (int i = 0; i < n; i++)
        if (a[i].numharm != b[i].numharm || a[i].harmnum != b[i].harmnum ||
            a[i].zmax != b[i].zmax || a[i].wmax != b[i].wmax || a[i].numz != b[i].numz ||
            a[i].numw != b[i].numw || a[i].fftlen != b[i].fftlen ||
            a[i].halfwidth != b[i].halfwidth)
            return 0;
    return 1;
}

static int resident_bank(const jerk_subharm *subs, int nsubs, void **bank)
{
    if (g_bank && g_bank_nsubs == nsubs && same_geometry(g_bank_subs, subs, nsubs)) {
        *bank = g_bank;
        return JERK_OK;
    }
    if (g_bank) {
        jerk_device_free(g_bank);
        free(g_bank_subs);
        g_bank = NULL;
        g_bank_subs = NULL;
    }
    void *b = NULL;
    int rc = jerk_device_alloc(8 * jerk_bank_elements(subs, nsubs), &b);
    if (rc == JERK_OK)
        rc = jerk_bank_generate(subs, nsubs, b, NULL);
    if (rc != JERK_OK) {
        if (b)
            jerk_device_free(b);
        return rc;
    }
    g_bank_subs = (jerk_subharm *)malloc(sizeof(jerk_subharm) * nsubs);
    memcpy(g_bank_subs, subs, sizeof(jerk_subharm) * nsubs);
    g_bank_nsubs = nsubs;
    g_bank = b;
    *bank = b;
    return JERK_OK;
}

static int gather_kernels(const subharminfo *s, float **out)
{
    const int fftlen = s->kern[0][0].fftlen;
    const size_t row = sizeof(fcomplex) * (size_t)fftlen;
    float *k = (float *)malloc(row * (size_t)s->numkern_wdim * s->numkern_zdim);
    if (!k)
        return -1;
    for (int ii = 0; ii < s->numkern_wdim; ii++)
        for (int jj = 0; jj < s->numkern_zdim; jj++)
            memcpy((char *)k + row * ((size_t)ii * s->numkern_zdim + jj), s->kern[ii][jj].data, row);
    *out = k;
    return 0;
}

int accelsearch_GPU(accelobs obs, subharminfo **subharminfs, GSList **cands_ptr, Cmdline *cmd)
{
    jerk_obs o;
    jerk_subharm *subs = NULL;
    float **kbufs = NULL;
    jerk_plan *plan = NULL;
    jerk_cand *cands = NULL;
    long long ncands = 0;
    int nsubs, rc = 0, idx = 0, gpu_bank = 0;
    void *bank = NULL;
    GSList *list = NULL;

    *cands_ptr = NULL;
    if (obs.inmem) {
        fprintf(stderr, "accelsearch_GPU: the in-memory search is not supported\n");
        rc = -1;
        goto done;
    }
    jerk_obs_of_accelobs(&obs, &o);

    nsubs = jerk_subharm_count(obs.numharmstages);
    subs = (jerk_subharm *)calloc(nsubs, sizeof(jerk_subharm));
    kbufs = (float **)calloc(nsubs, sizeof(float *));
    if (!subs || !kbufs) {
        rc = -1;
        goto done;
    }
    /* bank order (1/1), (1/2), (1/4), (3/4), ... as in fkern_host_to_dev
       (src/accel_utils_cu.c:378-429) */
    for (int stage = 0; stage < obs.numharmstages; stage++) {
        const int harmtosum = stage == 0 ? 2 : 1 << stage;
        for (int harm = 1; harm < harmtosum; harm += 2, idx++) {
            const subharminfo *s = &subharminfs[stage][harm - 1];
            jerk_subharm *d = &subs[idx];
            d->numharm = s->numharm;
            d->harmnum = s->harmnum;
            d->zmax = s->zmax;
            d->wmax = s->wmax;
            d->numz = s->numkern_zdim;
            d->numw = s->numkern_wdim;
            d->fftlen = s->kern[0][0].fftlen;
            d->halfwidth = s->kern[0][0].kern_half_width;
            if (!s->kern[0][0].data) {
                gpu_bank = 1;  /* the drop-in's create_subharminfos left the kernels out */
                continue;
            }
            if (gather_kernels(s, &kbufs[idx]) != 0) {
                rc = -1;
                goto done;
            }
            d->kernels = kbufs[idx];
        }
    }

    {
        jerk_config cfg;
        memset(&cfg, 0, sizeof(cfg));
        cfg.batch_rsteps = cmd && cmd->batchsize > 0 ? cmd->batchsize : 8;
        if (gpu_bank) {
            /* the kernel bank made on the GPU (src/accel_utils.c:151-282 restated
               in jerk_bank.cu) instead of uploaded from the host, kept for the
               next call of the same geometry */
            for (int i = 0; i < nsubs; i++)
                subs[i].kernels = NULL;
            rc = resident_bank(subs, nsubs, &bank);
            if (rc != JERK_OK) {
                fprintf(stderr, "accelsearch_GPU: %s\n", jerk_last_error());
                goto done;
            }
            cfg.device_bank = bank;
        }
        rc = jerk_plan_create(&plan, &o, subs, nsubs, &cfg);
        if (rc != JERK_OK) {
            fprintf(stderr, "accelsearch_GPU: %s\n", jerk_last_error());
            goto done;
        }
    }
    rc = jerk_search(plan, obs.fft, 0, 0, 0, &cands, &ncands, NULL);
    if (rc != JERK_OK) {
        fprintf(stderr, "accelsearch_GPU: %s\n", jerk_last_error());
        goto done;
    }
    /* the list in candidate order: prepend from the back */
    for (long long i = ncands - 1; i >= 0; i--) {
        accelcand *a = (accelcand *)malloc(sizeof(accelcand));
        a->power = cands[i].power;
        a->sigma = cands[i].sigma;
        a->numharm = cands[i].numharm;
        a->r = cands[i].r;
        a->z = cands[i].z;
        a->w = cands[i].w;
        a->pows = NULL;
        a->hirs = NULL;
        a->hizs = NULL;
        a->hiws = NULL;
        a->derivs = NULL;
        list = g_slist_prepend(list, a);
    }
    *cands_ptr = list;

done:
    if (plan)
        jerk_plan_destroy(plan);
    jerk_free(cands);
    if (kbufs)
        for (int i = 0; i < nsubs; i++)
            free(kbufs[i]);
    free(kbufs);
    free(subs);
    free_subharminfos(&obs, subharminfs);
    return rc == JERK_OK ? 0 : 1;
}
