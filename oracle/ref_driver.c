/*
 * Thin C-ABI driver over the REFERENCE's own accelsearch objects, compiled
 * from the reference sources by oracle/Makefile into oracle/_ref/.
 *
 * TEST INFRASTRUCTURE ONLY: tests/ and bench.py's CPU-baseline leg load the
 * resulting libprestoref.so through ctypes to (a) pin the oracle's
 * restatement against the reference itself and (b) time the reference CPU
 * search.  Nothing in the product links it.
 *
 * Every numeric result here comes from reference code:
 *   create_accelobs       src/accel_utils.c:1636-2037
 *   create_subharminfos   src/accel_utils.c:236-282
 *   subharm_fderivs_vol   src/accel_utils.c:1094-1293
 *   add_ffdotpows         src/accel_utils.c:1356-1377
 *   search_ffdotpows      src/accel_utils.c:1507-1555
 *   candidate_sigma, power_for_sigma   src/characteristics.c:647-705
 * The only logic of this file's own is ref_search's walk over the rsteps,
 * which has to be step-for-step the loop of src/accelsearch.c:183-223
 * (non-inmem path, add_ffdotpows) so that the candidate list it returns is
 * the one the reference's accelsearch builds before its optimisation stage.
 */
#include "accel.h"

#include <omp.h>
#include <stdlib.h>
#include <string.h>

typedef struct refctx {
    accelobs obs;
    infodata idata;
    Cmdline *cmd;      /* -> own_cmd */
    Cmdline own_cmd;   /* this context's parsed options */
    subharminfo **shis;
} refctx;

typedef struct ref_obs_summary {
    long long N, numbins, lobin, highestbin;
    int maxkernlen, corr_uselen, fftlen, numharmstages, numz, numw, norm_type, inmem;
    double dt, T, rlo, rhi, zlo, zhi, wlo, whi, nph;
    float powcut[6];
    long long numindep[6];
} ref_obs_summary;

typedef struct ref_cand {
    float power, sigma;
    int numharm;
    double r, z, w;
} ref_cand;

extern Cmdline *parseCmdline(int argc, char **argv);

/* The reference's parser (src/accelsearch_cmd.c:24, :1259) fills one
 * file-static Cmdline and never resets it, so an option given to one parse
 * (-locpow, -photon, ...) would stay set for every later one in this process.
 * Each open therefore restores the parser's defaults before parsing and keeps
 * its own copy of the result. */
static Cmdline *g_cmd_static;
static Cmdline g_cmd_defaults;

extern int get_birdies(char *zapfilenm, double T, double avg_vel, double **lobins,
                       double **hibins);
extern void zapbirds(double lobin, double hibin, FILE *fftfile, fcomplex *fft);

/* The step the reference's main takes between create_accelobs and the
 * kernels (src/accelsearch.c:85-107): with -zaplist and a spectrum held in
 * memory (a .dat input), the listed birdies are zapped in sorted order, the
 * list stopping at N/2 and a last birdie clamped below it. */
static void ref_zap_listed(refctx *c)
{
    if (!(c->cmd->zaplistP && !c->obs.mmap_file && c->obs.fft))
        return;
    double *lo, *hi;
    const int n = get_birdies(c->cmd->zaplist, c->obs.T, c->cmd->baryv, &lo, &hi);
    const double top = c->obs.N / 2;
    for (int ii = 0; ii < n; ii++) {
        if (lo[ii] >= top)
            break;
        if (hi[ii] >= top)
            hi[ii] = top - 1;
        zapbirds(lo[ii], hi[ii], NULL, c->obs.fft);
    }
    vect_free(lo);
    vect_free(hi);
}

refctx *ref_open(int argc, char **argv)
{
    refctx *c = (refctx *)calloc(1, sizeof(refctx));
    if (!g_cmd_static) {
        char prog[] = "accelsearch", file[] = "defaults.fft";
        char *a[] = {prog, file};
        g_cmd_static = parseCmdline(2, a);
        g_cmd_defaults = *g_cmd_static;
    }
    *g_cmd_static = g_cmd_defaults;
    c->own_cmd = *parseCmdline(argc, argv);
    c->cmd = &c->own_cmd;
    create_accelobs(&c->obs, &c->idata, c->cmd, 1);
    ref_zap_listed(c);
    return c;
}

void ref_get_obs(const refctx *c, ref_obs_summary *o)
{
    const accelobs *a = &c->obs;
    memset(o, 0, sizeof(*o));
    o->N = a->N;
    o->numbins = a->numbins;
    o->lobin = a->lobin;
    o->highestbin = a->highestbin;
    o->maxkernlen = a->maxkernlen;
    o->corr_uselen = a->corr_uselen;
    o->fftlen = a->fftlen;
    o->numharmstages = a->numharmstages;
    o->numz = a->numz;
    o->numw = a->numw;
    o->norm_type = a->norm_type;
    o->inmem = a->inmem;
    o->dt = a->dt;
    o->T = a->T;
    o->rlo = a->rlo;
    o->rhi = a->rhi;
    o->zlo = a->zlo;
    o->zhi = a->zhi;
    o->wlo = a->wlo;
    o->whi = a->whi;
    o->nph = a->nph;
    for (int ii = 0; ii < a->numharmstages && ii < 6; ii++) {
        o->powcut[ii] = a->powcut[ii];
        o->numindep[ii] = a->numindep[ii];
    }
}

void ref_make_bank(refctx *c)
{
    if (!c->shis)
        c->shis = create_subharminfos(&c->obs);
}

/* Subharmonic (stage, harm) with harm odd and < 2^stage (stage 0: harm 1).
 * info: numharm, harmnum, zmax, wmax, numkern_zdim, numkern_wdim, fftlen,
 *       kern_half_width of kern[0][0] */
int ref_shi_info(const refctx *c, int stage, int harm, int *info)
{
    const subharminfo *s;
    if (!c->shis)
        return -1;
    s = &c->shis[stage][harm - 1];
    info[0] = s->numharm;
    info[1] = s->harmnum;
    info[2] = s->zmax;
    info[3] = s->wmax;
    info[4] = s->numkern_zdim;
    info[5] = s->numkern_wdim;
    info[6] = s->kern[0][0].fftlen;
    info[7] = s->kern[0][0].kern_half_width;
    return 0;
}

/* Copy the kernel FFTs of one subharmonic, [w][z][fftlen] complex64. */
int ref_copy_kernels(const refctx *c, int stage, int harm, float *out)
{
    const subharminfo *s;
    if (!c->shis)
        return -1;
    s = &c->shis[stage][harm - 1];
    for (int ii = 0; ii < s->numkern_wdim; ii++)
        for (int jj = 0; jj < s->numkern_zdim; jj++) {
            const kernel *k = &s->kern[ii][jj];
            memcpy(out + 2L * ((long)ii * s->numkern_zdim + jj) * k->fftlen, k->data,
                   sizeof(fcomplex) * k->fftlen);
        }
    return 0;
}

/* One subharmonic ffdot volume for the rstep [fullrlo, fullrhi].
 * hdr: rlo, zlo, wlo, numrs, numzs, numws.  powers (if non-NULL) receives
 * numws*numzs*numrs floats; rinds/zinds (if non-NULL, numharm > 1) receive
 * corr_uselen / numz u16 entries. */
int ref_fderivs(refctx *c, int numharm, int harmnum, double fullrlo, double fullrhi,
                long long *hdr, float *powers, unsigned short *rinds,
                unsigned short *zinds)
{
    int stage = 0;
    subharminfo *s;
    ffdotpows *f;
    while ((1 << stage) < numharm)
        stage++;
    ref_make_bank(c);
    s = &c->shis[stage][harmnum - 1];
    f = subharm_fderivs_vol(numharm, harmnum, fullrlo, fullrhi, s, &c->obs);
    hdr[0] = f->rlo;
    hdr[1] = f->zlo;
    hdr[2] = f->wlo;
    hdr[3] = f->numrs;
    hdr[4] = f->numzs;
    hdr[5] = f->numws;
    if (powers)
        memcpy(powers, f->powers[0][0],
               sizeof(float) * (size_t)f->numws * f->numzs * f->numrs);
    if (numharm > 1 && rinds)
        memcpy(rinds, f->rinds, sizeof(unsigned short) * c->obs.corr_uselen);
    if (numharm > 1 && zinds)
        memcpy(zinds, f->zinds, sizeof(unsigned short) * c->obs.numz);
    free_ffdotpows(f);
    return 0;
}

/* The reference search over at most max_steps rsteps starting at obs.rlo
 * (all of them if max_steps <= 0).  Returns the number of candidates in the
 * final list (copied in list order into out, up to max_out), or -1. */
long ref_search(refctx *c, long max_steps, ref_cand *out, long max_out, long *steps_done)
{
    GSList *cands = NULL, *lp;
    double startr, lastr, nextr;
    int rstep = c->obs.corr_uselen * ACCEL_DR;
    long nsteps = 0, ncand = 0;
    accelobs *obs = &c->obs;

    if (obs->inmem)
        return -1;
    ref_make_bank(c);
    startr = obs->rlo;
    while (startr + rstep < obs->highestbin && (max_steps <= 0 || nsteps < max_steps)) {
        ffdotpows *fundamental;
        nextr = startr + rstep;
        lastr = nextr - ACCEL_DR;
        fundamental = subharm_fderivs_vol(1, 1, startr, lastr, &c->shis[0][0], obs);
        cands = search_ffdotpows(fundamental, 1, obs, cands);
        if (obs->numharmstages > 1) {
            for (int stage = 1; stage < obs->numharmstages; stage++) {
                int harmtosum = 1 << stage;
                for (int harm = 1; harm < harmtosum; harm += 2) {
                    ffdotpows *sub = subharm_fderivs_vol(harmtosum, harm, startr, lastr,
                                                         &c->shis[stage][harm - 1], obs);
                    add_ffdotpows(fundamental, sub, harmtosum, harm);
                    free_ffdotpows(sub);
                }
                cands = search_ffdotpows(fundamental, harmtosum, obs, cands);
            }
        }
        free_ffdotpows(fundamental);
        startr = nextr;
        nsteps++;
    }
    for (lp = cands; lp; lp = lp->next, ncand++) {
        if (ncand < max_out && out) {
            accelcand *a = (accelcand *)lp->data;
            out[ncand].power = a->power;
            out[ncand].sigma = a->sigma;
            out[ncand].numharm = a->numharm;
            out[ncand].r = a->r;
            out[ncand].z = a->z;
            out[ncand].w = a->w;
        }
    }
    g_slist_foreach(cands, free_accelcand, NULL);
    g_slist_free(cands);
    if (steps_done)
        *steps_done = nsteps;
    return ncand;
}

/* Feed a hit sequence, one hit per call, through the reference's own
 * search_ffdotpows (and so its static insert_new_accelcand): each hit is a
 * 1x1x1 volume at fundamental bin rlo[i] with power pows[i], searched as
 * numharm[i] summed harmonics.  Powers must exceed obs.powcut of their stage.
 * Returns the final list like ref_search. */
long ref_insert_sequence(refctx *c, long n, const float *pows, const long long *rlo,
                         const int *numharm, ref_cand *out, long max_out)
{
    GSList *cands = NULL, *lp;
    long ncand = 0;
    float *cell = gen_fvect(1);
    float *rows[1] = {cell};
    float **planes[1] = {rows};
    for (long i = 0; i < n; i++) {
        ffdotpows f;
        memset(&f, 0, sizeof(f));
        f.rlo = rlo[i];
        f.zlo = 0;
        f.wlo = 0;
        f.numrs = f.numzs = f.numws = 1;
        f.powers = planes;
        cell[0] = pows[i];
        cands = search_ffdotpows(&f, numharm[i], &c->obs, cands);
    }
    vect_free(cell);
    for (lp = cands; lp; lp = lp->next, ncand++) {
        if (ncand < max_out && out) {
            accelcand *a = (accelcand *)lp->data;
            out[ncand].power = a->power;
            out[ncand].sigma = a->sigma;
            out[ncand].numharm = a->numharm;
            out[ncand].r = a->r;
            out[ncand].z = a->z;
            out[ncand].w = a->w;
        }
    }
    g_slist_foreach(cands, free_accelcand, NULL);
    g_slist_free(cands);
    return ncand;
}

double ref_candidate_sigma(double power, int numsum, double numtrials)
{
    return candidate_sigma(power, numsum, numtrials);
}

double ref_power_for_sigma(double sigma, int numsum, double numtrials)
{
    return power_for_sigma(sigma, numsum, numtrials);
}

int ref_w_resp_halfwidth(double z, double w, int highacc)
{
    return w_resp_halfwidth(z, w, highacc ? HIGHACC : LOWACC);
}

int ref_next_good_fftlen(int n) { return next_good_fftlen(n); }

int ref_fftlen_from_kernwidth(int kernwidth) { return fftlen_from_kernwidth(kernwidth); }

float ref_median(float *arr, int n) { return median(arr, n); }

/* The reference's local power levels (src/corr_routines.c:309-366) and its
 * fast inverse square root (src/misc_utils.c:293-304), for pinning the
 * -locpow normalisation. */
void ref_corr_loc_pow(float *powers, int n, float *out)
{
    float *lp = corr_loc_pow(powers, n);
    memcpy(out, lp, sizeof(float) * n);
    vect_free(lp);
}

float ref_invsqrtf(float x) { return invsqrtf(x); }

/* The reference's kernel response for one (z, w), before placement and FFT:
 * numkern complex64 values from gen_w_response (src/responses.c:333-418). */
int ref_gen_w_response(double roffset, int numbetween, double z, double w, int numkern,
                       float *out)
{
    fcomplex *r = gen_w_response(roffset, numbetween, z, w, numkern);
    memcpy(out, r, sizeof(fcomplex) * numkern);
    vect_free(r);
    return 0;
}

/* OpenMP threads used by the reference's parallel loops; the reference's own
 * main sets 1 unless -ncpus asks for more (src/accelsearch.c:120-131), and
 * only the single-thread order of insertions is deterministic. */
void ref_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }

/* The reference's candidate optimisation (optimize_accelcand,
 * src/accel_utils.c:573-657) of one candidate; obs must hold the spectrum in
 * memory (a .dat input or a memory-mapped .fft).  out receives, per
 * harmonic h: pows, hirs, hizs, hiws and the 7 doubles of rderivs (pow,
 * phs, dpow, dphs, d2pow, d2phs, locpow), 11 doubles each; *sigma the
 * recomputed sigma.  Returns 0, or -1 without a spectrum in memory. */
int ref_optimize_cand(refctx *c, float power, int numharm, double r, double z, double w,
                      double *out, float *sigma)
{
    if (!c->obs.fft)
        return -1;
    accelcand cand;
    memset(&cand, 0, sizeof(cand));
    cand.power = power;
    cand.numharm = numharm;
    cand.r = r;
    cand.z = z;
    cand.w = w;
    optimize_accelcand(&cand, &c->obs);
    for (int h = 0; h < numharm; h++) {
        double *o = out + 11 * h;
        o[0] = cand.pows[h];
        o[1] = cand.hirs[h];
        o[2] = cand.hizs[h];
        o[3] = cand.hiws[h];
        o[4] = cand.derivs[h].pow;
        o[5] = cand.derivs[h].phs;
        o[6] = cand.derivs[h].dpow;
        o[7] = cand.derivs[h].dphs;
        o[8] = cand.derivs[h].d2pow;
        o[9] = cand.derivs[h].d2phs;
        o[10] = cand.derivs[h].locpow;
    }
    *sigma = cand.sigma;
    free(cand.pows);
    free(cand.hirs);
    free(cand.hizs);
    free(cand.hiws);
    free(cand.derivs);
    return 0;
}

/* The reference's harmonic polishing volume search (max_rzw_arr_harmonics,
 * src/maximize_rzw.c:84-190) for a candidate at (rin, zin, win), rin
 * relative to obs.lobin: rzw[0..2] = polished r, z, w; locpow[i] = the float
 * local power of harmonic n = numharm - i that it divides by
 * (get_localpower3d, src/characteristics.c:75-135).  -1 without a spectrum
 * in memory. */
int ref_polish(refctx *c, int numharm, double rin, double zin, double win, double *rzw,
               float *locpow)
{
    if (!c->obs.fft)
        return -1;
    rderivs *d = (rderivs *)malloc(sizeof(rderivs) * numharm);
    double *pows = (double *)malloc(sizeof(double) * numharm);
    for (int i = 0; i < numharm; i++) {
        const int n = numharm - i;
        locpow[i] = (float)get_localpower3d(c->obs.fft, c->obs.numbins, rin * n, zin * n,
                                            win * n);
    }
    max_rzw_arr_harmonics(c->obs.fft, c->obs.numbins, numharm, rin, zin, win, rzw, rzw + 1,
                          rzw + 2, d, pows);
    free(d);
    free(pows);
    return 0;
}

/* The spectrum the reference searches, when it holds one in memory: a .dat
 * input after its realfft and deredden (src/accel_utils.c:1696-1753), or a
 * memory-mapped .fft.  Copies up to max complex values; -1 if none. */
long ref_copy_spectrum(const refctx *c, float *out, long max)
{
    if (!c->obs.fft)
        return -1;
    long n = c->obs.numbins < max ? c->obs.numbins : max;
    memcpy(out, c->obs.fft, sizeof(fcomplex) * (size_t)n);
    return n;
}

void ref_close(refctx *c)
{
    if (!c)
        return;
    if (c->shis)
        free_subharminfos(&c->obs, c->shis);
    free_accelobs(&c->obs);
    free(c);
}
