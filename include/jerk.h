/*
 * libjerk: B200 (sm_100a) Fourier-domain jerk search -- the C ABI.
 *
 * Drop-in for the search loop of PrestoZL's accelsearch_cu: everything
 * between the reference's accelsearch_CPU1 (command line, accelobs, kernel
 * bank) and accelsearch_CPU2 (sort, harmonic elimination, optimisation,
 * ACCEL output) runs here on the GPU.  Plain pointers and sizes only.
 *
 * Reference interfaces each entry point replaces (paths inside the
 * reference project):
 *   jerk_plan_create   accelsearch_GPU set-up: init_constant_device,
 *                      fkern_host_to_dev, buffer sizing
 *                      (src/accelsearch_lib.c:473-645,
 *                       src/accel_kernels.cu:73-79,
 *                       src/accel_utils_cu.c:378-429)
 *   jerk_search        accelsearch_GPU's batch loop + insert_to_cands
 *                      (src/accelsearch_lib.c:660-878,
 *                       src/accel_utils_cu.c:432-612 do_fft_batch /
 *                       fuse_add_search_batch / sort_search_results,
 *                       src/accel_utils_cu.c:857-929)
 *   jerk_plan_destroy  accelsearch_GPU tear-down (cudaFree*, clear_cache;
 *                      src/accelsearch_lib.c:866-878)
 *   jerk_obs_from_params / jerk_subharm_sizes
 *                      the sizing part of create_accelobs and
 *                      init_subharminfo (src/accel_utils.c:1795-2004,
 *                      199-234, 137-149)
 *   jerk_candidate_sigma / jerk_power_for_sigma
 *                      candidate_sigma / power_for_sigma
 *                      (src/characteristics.c:647-705)
 *   jerk_bank_generate the kernel bank of create_subharminfos
 *                      (src/accel_utils.c:151-282, src/responses.c:333-418)
 *   jerk_polish_rzw / jerk_optimize_cand / jerk_local_power / jerk_derivs
 *                      optimize_accelcand's harmonic polishing
 *                      (src/accel_utils.c:573-657, src/maximize_rzw.c:84-190,
 *                       get_localpower3d / get_derivs3d
 *                       src/characteristics.c:75-191)
 *   jerk_realfft / jerk_deredden / jerk_spectrum_from_timeseries /
 *   jerk_zap_birdies   the .dat input of create_accelobs and CPU1's zapping
 *                      (src/fastffts.c:163-235, src/accel_utils.c:1557-1633,
 *                       1696-1753, src/accelsearch_lib.c:393-418)
 *   jerk_downsample_subbands / jerk_dedisp_subbands
 *                      prepsubband_cu's DownsampDataArray / getDedisp
 *                      (src/prepsubband_kernels.cu:21-87)
 *   jerk_server_*      the served form (no counterpart in the reference)
 *
 * Return codes: JERK_OK, > 0 recoverable, < 0 fatal (no exit() anywhere).
 */
#ifndef JERK_H
#define JERK_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define JERK_OK 0
#define JERK_OVERFLOW 1          /* more hits than the hit buffer holds; retried internally */
#define JERK_TIMEOUT 2           /* a bounded wait gave up */
#define JERK_EINVAL (-1)         /* bad argument */
#define JERK_ECUDA (-2)          /* CUDA runtime error */
#define JERK_ENOMEM (-3)         /* device or host allocation failed */
#define JERK_EUNSUPPORTED (-4)   /* a configuration the engine does not handle */

#define JERK_MAX_STAGES 6

/* The search geometry of one spectrum: the fields of the reference's
 * accelobs (include/accel.h:37-82) that the search loop reads. */
typedef struct jerk_obs {
    long long numbins;        /* complex bins in the spectrum */
    long long lobin;          /* bin number of spectrum[0] */
    long long highestbin;     /* the search stops before this bin */
    double rlo;               /* first fundamental Fourier bin searched */
    double zlo;               /* -zmax */
    double wlo;               /* -wmax */
    int corr_uselen;          /* good interbins per rstep */
    int numz;                 /* fundamental f-dot count */
    int numw;                 /* accelobs.numw (0 when -wmax 0) */
    int numharmstages;        /* log2(numharm) + 1 */
    int norm_type;            /* 0: block median; 1: local power (-locpow);
                                 ignored when nph > 0 (-photon) */
    float nph;                /* > 0: photon normalisation */
    float powcut[JERK_MAX_STAGES];
    long long numindep[JERK_MAX_STAGES];
} jerk_obs;

/* One subharmonic's kernel set (the reference's subharminfo,
 * include/accel.h:110-122). */
typedef struct jerk_subharm {
    int numharm, harmnum;     /* harmonic fraction harmnum/numharm */
    int zmax, wmax;           /* this subharmonic's own maxima */
    int numz, numw;           /* numkern_zdim, numkern_wdim */
    int fftlen;
    int halfwidth;            /* kern[0][0].kern_half_width */
    const void *kernels;      /* host complex64 [numw][numz][fftlen], or NULL
                                 with a device bank (jerk_config.device_bank) */
} jerk_subharm;

/* A candidate: the leading fields of the reference's accelcand
 * (include/accel.h:84-97). */
typedef struct jerk_cand {
    float power;
    float sigma;
    int numharm;
    double r, z, w;
} jerk_cand;

typedef struct jerk_config {
    int batch_rsteps;         /* rsteps per batch (the reference's -batchsize); 0 = 8;
                                 capped to what 32-bit volume offsets allow */
    long long max_hits;       /* initial hit-buffer capacity; 0 = auto */
    void *stream;             /* cudaStream_t to run on; NULL = a private stream */
    const void *device_bank;  /* optional resident bank (jerk_bank_generate); it
                                 must be complete when the plan is created (the
                                 plan folds its fftlen-2048 and -1280 rows from it
                                 then) */
    int harm_mode;            /* harmonic-sum kernel (a tuning knob; results do
                                 not depend on it): 1 = gather (global loads),
                                 2 = gather + TMA prefetch of the next tile into
                                 L2, 3 / 4 = TMA copies of 8 / 16-row tiles into
                                 shared memory (modes 2-4 fall back to 1 where
                                 tensor maps cannot be built); 0 = 1 */
    int use_graph;            /* nonzero: each jerk_search / jerk_search_async
                                 pass is captured once per (first_rstep,
                                 num_rsteps) into a CUDA graph and replayed for
                                 later spectra (the spectrum is staged into a
                                 plan buffer first); 0 = launch batch by batch */
} jerk_config;

typedef struct jerk_plan jerk_plan;

/* Raw threshold crossings of one search, in the reference's insertion order
 * (rstep, stage, w, z, r). */
typedef struct jerk_hits {
    long long count;
    unsigned long long *keys; /* encoded (rstep, stage, w, z, r) */
    float *powers;
} jerk_hits;

int jerk_obs_from_params(long long numbins, long long N, double dt, int zmax, int wmax,
                         int wmax_given, int numharm, float sigma, double flo, double fhi,
                         jerk_obs *obs, int *fftlen, int *maxkernlen);
int jerk_subharm_count(int numharmstages);
int jerk_subharm_sizes(const jerk_obs *obs, int fftlen, int index, jerk_subharm *out);

int jerk_plan_create(jerk_plan **plan, const jerk_obs *obs, const jerk_subharm *subs,
                     int nsubs, const jerk_config *cfg);
void jerk_plan_destroy(jerk_plan *plan);

/* Search rsteps [first_rstep, first_rstep + num_rsteps) (num_rsteps <= 0:
 * to the end).  spectrum: numbins complex64, on the host (copied in) or on
 * the device (spectrum_on_device != 0).  The final candidate list (the
 * reference's GSList contents, in list order) is written to *cands, which the
 * caller frees with jerk_free; hits (optional) receives the raw crossings. */
int jerk_search(jerk_plan *plan, const void *spectrum, int spectrum_on_device,
                long long first_rstep, long long num_rsteps, jerk_cand **cands,
                long long *ncands, jerk_hits *hits);

/* The same search in parts, so one host thread can keep several plans busy:
 * jerk_search_async stages the spectrum and enqueues the first few batches;
 * jerk_search_advance(plan, ahead) enqueues more while fewer than `ahead`
 * batches are queued or running (returns 1 while batches remain, 0 once all
 * are enqueued); jerk_search_ready reports without blocking whether all the
 * device work is done (1), not yet (0) or failed (< 0); jerk_search_collect
 * enqueues whatever remains, waits, and builds the candidate list.  One
 * search in flight per plan; a host spectrum must stay valid until collect. */
int jerk_search_async(jerk_plan *plan, const void *spectrum, int spectrum_on_device,
                      long long first_rstep, long long num_rsteps);
int jerk_search_advance(jerk_plan *plan, int ahead);
int jerk_search_ready(jerk_plan *plan);
int jerk_search_collect(jerk_plan *plan, jerk_cand **cands, long long *ncands, jerk_hits *hits);

/* The batched form across plans: several searches (spectra of any length,
 * plans of any geometry) advanced in waves of merged launches.  One wave
 * takes the next batch of every listed plan with work left (up to 12 per
 * wave) and runs one prep launch, one correlation launch per FFT length and
 * one harmonic-sum launch per stage count over all of them, so small
 * searches share the GPU instead of each underfilling it.  Each plan's
 * results are bitwise those of jerk_search.  Replaces, for this purpose, the
 * reference's process pool (bin/accelsearch_pipeline_cu.py:296-407), whose
 * processes each run their own batches (src/accelsearch_lib.c:660-830).
 *   jerk_search_begin    stages the spectrum and starts a pass without
 *                        enqueueing anything (no graph replay);
 *   jerk_group_advance   enqueues waves while the listed plans have fewer
 *                        than `ahead` batches queued or running (ahead <= 0:
 *                        everything); the plans whose passes are in flight
 *                        must share one stream and device.  Returns 1 while
 *                        batches remain, 0 once all are enqueued, < 0 on error;
 *   then jerk_search_ready / jerk_search_collect per plan as above;
 *   jerk_search_group    all of it for whole spectra: begin, advance
 *                        everything, collect; cands[i] / ncands[i] receive
 *                        plan i's list (free each with jerk_free). */
int jerk_search_begin(jerk_plan *plan, const void *spectrum, int spectrum_on_device,
                      long long first_rstep, long long num_rsteps);
int jerk_group_advance(jerk_plan *const *plans, int nplans, int ahead);
int jerk_search_group(jerk_plan *const *plans, const void *const *spectra,
                      const int *spectrum_on_device, int nplans, jerk_cand **cands,
                      long long *ncands);

/* Device memory the plan holds (volumes, tables, hit buffer, its own bank). */
long long jerk_plan_device_bytes(const jerk_plan *plan);

/* Number of rsteps of the full search. */
long long jerk_num_rsteps(const jerk_plan *plan);

/* Debug/test: the ffdot volume of subharmonic 'sub' at rstep 'rstep'
 * ([numw][numz][numrs] floats, numrs written to *numrs). */
int jerk_debug_volume(jerk_plan *plan, const void *spectrum, int spectrum_on_device,
                      long long rstep, int sub, float *out, int *numrs, long long *rlo);

/* Debug/test: with on != 0, every later pass of the plan also runs one
 * bounded wait that must give up (the correlation's bounded mbarrier wait, in
 * a one-thread kernel on the plan's stream, on an mbarrier that nothing
 * completes; no copy is involved).  The pass then fails with JERK_ECUDA, as a
 * data-row copy that never completes would, and the plan stays usable.  The reference has no bounded waits: its CUDA errors
 * exit the process (include/cuda_helper.h:2-16). */
int jerk_debug_wait_probe(jerk_plan *plan, int on);

/* Instrumentation.  Every launch is counted with its algorithmic bytes and
 * flops; with profiling on, each launch is also bracketed by CUDA events on
 * the plan's stream and its device time accumulated per kernel class
 * ("prep", "corr_<fftlen>", "harmsum"). */
typedef struct jerk_kernel_stat {
    char name[32];
    long long launches;
    double ms;                /* summed device time (profiling on) */
    double bytes;             /* summed algorithmic bytes */
    double flops;             /* summed algorithmic flops */
} jerk_kernel_stat;

int jerk_plan_set_profiling(jerk_plan *plan, int on);
void jerk_plan_reset_stats(jerk_plan *plan);
/* Number of kernel classes; fills up to max entries of out. */
int jerk_plan_kernel_stats(const jerk_plan *plan, int max, jerk_kernel_stat *out);
/* Bytes copied host->device (spectra) and device->host (hit lists). */
void jerk_plan_transfer_stats(const jerk_plan *plan, long long *h2d, long long *d2h);

/* Kernel bank on the device: [sub][w][z][fftlen] complex64 for the given
 * subharmonics (in jerk_subharm_sizes order), the layout jerk_plan_create
 * takes as jerk_config.device_bank.  device_bank must hold
 * jerk_bank_elements() complex64 values; stream may be NULL. */
long long jerk_bank_elements(const jerk_subharm *subs, int nsubs);
/* cudaMalloc / cudaFree for callers without their own device allocator. */
int jerk_device_alloc(long long bytes, void **out);
void jerk_device_free(void *p);
int jerk_copy_to_host(void *dst, const void *device_src, long long bytes);
int jerk_bank_generate(const jerk_subharm *subs, int nsubs, void *device_bank, void *stream);

/* One subharmonic's ffdot volume for one rstep without allocating anything.
 * No counterpart in the reference: it exists for callers that cannot
 * allocate device memory when they search (memory handed out up front by a
 * pool they do not own, real-time loops that forbid allocation after
 * start-up).  All working memory is a fixed 192 KiB device array inside the
 * library (fftlen <= 7680, corr_uselen <= 16384; larger sizes are rejected
 * with JERK_EINVAL).  spectrum (numbins complex64, bin 0 = lobin), kernels
 * (this subharmonic's [numw][numz][fftlen] rows) and volume
 * ([numw][numz][numrs] floats, numrs <= corr_uselen + 8 is enough) are
 * device pointers owned by the caller; fullrlo is the rstep's first
 * fundamental r.  Normalisation is the block median, or 1/sqrt(nph) when
 * nph > 0 (-photon); the local-power normalisation of -locpow is not
 * offered here (use a plan).  The call only launches kernels on stream
 * (NULL = default stream): descriptors go as kernel parameters and the FFT
 * twiddles are computed on the device, so nothing is copied from host
 * memory.  The first call on each device looks the array up
 * (cudaGetSymbolAddress): make it before any stream capture.  Calls share
 * the array, so calls that overlap on the GPU race; serialise them.
 * Failures set jerk_last_error. */
int jerk_volume_static(const void *spectrum, long long numbins, long long lobin,
                       const jerk_subharm *sub, const void *kernels, double fullrlo,
                       int corr_uselen, float nph, float *volume, int *numrs, long long *rlo,
                       void *stream);

/* Candidate polishing on the GPU: the volume search of the reference's
 * harmonic polishing, max_rzw_arr_harmonics (src/maximize_rzw.c:84-190),
 * which optimize_accelcand (src/accel_utils.c:573-657) runs for every final
 * candidate of a search with -wmax.  Per harmonic n = numharm .. 1 it
 * correlates the spectrum with 17 x 17 (z, w) responses at 8 points per bin
 * around (n r, n z, n w), sums |amplitude|^2 / locpow over the harmonics and
 * takes the first strict maximum; *rout, *zout, *wout are the polished
 * fundamental values as the reference computes them, *maxpow the summed
 * power there.
 *   spectrum  numdata complex64 values (the searched spectrum; value 0 is
 *             obs.lobin), read around each harmonic only: on the host (the
 *             reference's obs->fft), or in device memory, where a kernel
 *             gathers the windows and nothing of the spectrum crosses PCIe
 *             (the polisher asks the driver which; a device spectrum must be
 *             complete when the call is made, or written on its stream).
 *             The same holds for jerk_local_power, jerk_derivs and
 *             jerk_optimize_cand below.
 *   rin       the candidate's r minus obs.lobin; zin, win its z and w
 *   locpow    numharm floats: get_localpower3d (src/characteristics.c:75-135)
 *             of harmonic n = numharm - i at (n rin, n zin, n win), as float
 * A jerk_polisher holds the device buffers (grown to the largest candidate)
 * and runs on its stream (NULL: its own); one call at a time per polisher.
 * Correlation or response FFTs longer than 8192 points (about zmax 300 with
 * wmax 600 and above) return JERK_EUNSUPPORTED.  Not in the reference: the
 * reference runs this on the CPU, one candidate after another. */
typedef struct jerk_polisher jerk_polisher;
int jerk_polisher_create(jerk_polisher **polisher, void *stream);
void jerk_polisher_destroy(jerk_polisher *polisher);
int jerk_polish_rzw(jerk_polisher *polisher, const void *spectrum, long long numdata, int numharm,
                    double rin, double zin, double win, const float *locpow, double *rout,
                    double *zout, double *wout, float *maxpow);

/* The reference's rderivs (include/presto.h:161-169): power and phase at a
 * point of the f / f-dot / f-dotdot volume, their first and second
 * derivatives in r, and the local power level. */
typedef struct jerk_rderivs {
    double pow, phs, dpow, dphs, d2pow, d2phs, locpow;
} jerk_rderivs;

/* get_localpower3d (src/characteristics.c:75-135) at n points (r relative
 * to the spectrum's value 0): the mean power of the complex interpolations
 * (rzw_interp, src/rzwinterp.c:151-228) at the 10 bins either side, 5 bins
 * away.  On the GPU; results agree with the reference's to FP32 rounding. */
int jerk_local_power(jerk_polisher *polisher, const void *spectrum, long long numdata, int n,
                     const double *r, const double *z, const double *w, double *out);
/* get_derivs3d (src/characteristics.c:138-191) at n points with the given
 * local powers: interpolations 0.003 bins apart at HIGHACC, then the finite
 * differences of power and phase. */
int jerk_derivs(jerk_polisher *polisher, const void *spectrum, long long numdata, int n,
                const double *r, const double *z, const double *w, const double *locpow,
                jerk_rderivs *out);
/* The reference's default candidate optimisation (optimize_accelcand with
 * harmonic polishing, src/accel_utils.c:573-657) wholly on the GPU: local
 * powers, jerk_polish_rzw, then per harmonic h = 1..numharm the local power
 * and derivatives at (h r, h z, h w).  rzw_out[3] = polished r (relative to
 * value 0), z, w; derivs[numharm]; locpow_used[numharm] (optional) = the local
 * powers the volume search divided by.  Without the reference's host
 * routines the derivatives agree with its to FP32 rounding (the drop-in
 * keeps the reference's own routines for byte-identical ACCEL files). */
int jerk_optimize_cand(jerk_polisher *polisher, const void *spectrum, long long numdata,
                       int numharm, double rin, double zin, double win, double *rzw_out,
                       jerk_rderivs *derivs, float *locpow_used);

/* The search's input from a time series, on the GPU: the steps the reference
 * takes for a ".dat" input (src/accel_utils.c:1696-1753) before it searches.
 *
 * jerk_realfft replaces realfft(idata, n, -1) (src/fastffts.c:163-235): the
 * forward real FFT of n float samples, unnormalised, packed as the reference
 * packs it -- n/2 complex64 values, value 0 = (DC, Nyquist), value k = bin k.
 * n must be 2 R1 R2 with R1, R2 in {128, 192, 256, 384, 512, 768, 1024, 1280,
 * 2048, 4096, 5120, 7680, 8192, 10240} -- powers of two from 2^15 to 2^27
 * and lengths with factors 3 and 5 such as 3 * 2^20 or 15 * 2^20
 * (JERK_EUNSUPPORTED otherwise; jerk_realfft_scratch_bytes returns 0).
 * FP32 like the reference's, so results agree to FP32 rounding.
 *
 * jerk_deredden replaces deredden(fft, numamps) (src/accel_utils.c:1557-1633)
 * in place on numamps complex64 values (8 <= numamps < 2^31), bit-exact with
 * the reference.
 *
 * jerk_spectrum_from_timeseries runs both and then sets bin 0 to (1, 1), as
 * create_accelobs prepares a .dat input searched without -photon
 * (src/accel_utils.c:1747-1753, 1829-1834).
 *
 * All pointers are device pointers owned by the caller: the series and the
 * spectrum 8-byte aligned (they may be the same buffer: n floats = n/2
 * complex64), scratch 256-byte aligned and at least the matching
 * *_scratch_bytes (0 = size not supported).  Asynchronous on stream
 * (NULL = default stream); nothing is allocated. */
long long jerk_realfft_scratch_bytes(long long n);
int jerk_realfft(const float *timeseries, long long n, void *spectrum, void *scratch,
                 long long scratch_bytes, void *stream);
long long jerk_deredden_scratch_bytes(long long numamps);
int jerk_deredden(void *spectrum, long long numamps, void *scratch, long long scratch_bytes,
                  void *stream);
/* Birdie zapping of the spectrum made from a time series, replacing the
 * loop of src/accelsearch_lib.c:393-418 over zapbirds (src/zapping.c:29-81,
 * from memory): for each birdie [lobins[i], hibins[i]] in Fourier bins, in
 * list order (stopping at the first at or above N/2, high edges clamped to
 * N/2 - 1), the bins [floor(lo), ceil(hi)) take the amplitude
 * sqrt(0.5 (median power of the 200 bins from lo - 300 + median power of the
 * 200 bins from hi - 100) / ln 2) with phase 0; birdies below 301 bins are
 * left alone.  Bit-exact with the reference.  spectrum: numbins complex64 on
 * the device; lobins/hibins: host arrays (the reference's get_birdies
 * output).  Asynchronous on stream; allocates nothing. */
int jerk_zap_birdies(void *spectrum, long long numbins, long long N, const double *lobins,
                     const double *hibins, int nbirds, void *stream);
long long jerk_spectrum_scratch_bytes(long long n);
int jerk_spectrum_from_timeseries(const float *timeseries, long long n, void *spectrum,
                                  void *scratch, long long scratch_bytes, void *stream);

/* Subband dedispersion: the GPU steps of prepsubband_cu, which makes the DM
 * trials' time series that the search takes (src/prepsubband_cu.c:1140-1165).
 * Data are blocks of worklen samples of nsub subbands, time-major
 * ([t][s], subband fastest), float32, on the device.
 *
 * jerk_downsample_subbands replaces DownsampDataArray
 * (src/prepsubband_kernels.cu:23-46, 76-80): out[t][s] = the mean of
 * in[t bs + k][s] over k < bs, for t < worklen (the output length).
 *
 * jerk_dedisp_subbands replaces getDedisp (src/prepsubband_kernels.cu:48-74,
 * 82-87; the CPU form float_dedisp, src/dispersion.c:208-231): out[dm][t]
 * (numdms rows of worklen) = the sum over s of x[t + offsets[dm][s]][s], where
 * x is last (the previous block) followed by cur (this one).  The offsets
 * (prepsubband_cu's offsets[numdms][nsub], in downsampled samples, each in
 * [0, worklen]) are fixed for a run, so they are given once, on the host or
 * the device (getDedisp's offsets_gpu), to jerk_dedisperser_create, which
 * checks them and plans the tiling.  jerk_dedisperser_matches returns 1 when
 * a dedisperser was made for these sizes and offsets.
 *
 * Both sum in the reference's order in FP32, bit-exact with the reference.
 * Asynchronous on stream (NULL: the legacy default stream, as the reference
 * launches); no allocation per call. */
int jerk_downsample_subbands(float *out, const float *in, int worklen, int bs, int nsub,
                             void *stream);
typedef struct jerk_dedisperser jerk_dedisperser;
int jerk_dedisperser_create(jerk_dedisperser **dedisperser, int worklen, int nsub, int numdms,
                            const int *offsets);
void jerk_dedisperser_destroy(jerk_dedisperser *dedisperser);
/* the tiling chosen: DMs per CTA group and samples per tile */
int jerk_dedisperser_shape(const jerk_dedisperser *dedisperser, int *group_dms, int *tile_samples);
/* Host only (no CUDA call): the checks and the tiling choice of
 * jerk_dedisperser_create for a host offsets table, with the shared memory a
 * CTA takes. */
int jerk_dedisp_plan(int worklen, int nsub, int numdms, const int *offsets, int *group_dms,
                     int *tile_samples, long long *smem_bytes);
int jerk_dedisperser_matches(const jerk_dedisperser *dedisperser, int worklen, int nsub, int numdms,
                             const int *offsets);
int jerk_dedisp_subbands(jerk_dedisperser *dedisperser, const float *cur, const float *last,
                         float *out, void *stream);

/* The served form: a request loop on one GPU (continuous batching).
 * Submitted spectra wait in a queue; a worker thread that owns the device
 * admits them while fewer than max_active searches run and their device
 * footprint fits hbm_budget_bytes, keeps the admitted searches in flight
 * together -- their batches run in waves of merged launches on the server's
 * stream (jerk_group_advance), so a request admitted while others run shares
 * their launches from its next wave on -- and queues each finished
 * candidate list for jerk_server_poll.  Kernel banks are generated once per search geometry and
 * shared; idle plans of the same geometry are reused.  A result equals
 * jerk_search's for the same spectrum and parameters.  (The reference's
 * counterpart is the process pool of bin/accelsearch_pipeline_cu.py.) */
typedef struct jerk_server jerk_server;

typedef struct jerk_server_config {
    long long hbm_budget_bytes;  /* admission budget; 0 = 85% of free device memory */
    int max_active;              /* searches in flight at once; 0 = 3 */
    int batch_rsteps;            /* rsteps per batch of each plan; 0 = 16 */
    int device;                  /* CUDA device the worker owns */
    int batches_ahead;           /* waves each search keeps queued; 0 = 3 */
    double queue_timeout_s;      /* a request not admitted within this fails
                                    with JERK_TIMEOUT; 0 = never */
    int harm_mode;               /* jerk_config.harm_mode of every plan */
} jerk_server_config;

typedef struct jerk_request {
    const void *spectrum;        /* numbins complex64; valid until its result is polled */
    int on_device;               /* spectrum is a device pointer */
    long long numbins;
    long long N;                 /* time samples (the .inf's N) */
    double dt;
    int zmax, wmax, wmax_given, numharm;
    float sigma;
    double flo, fhi;             /* accelsearch's -flo / -fhi (defaults 1, 10000) */
    long long tag;               /* the caller's id, returned with the result */
    int timeseries;              /* nonzero: `spectrum` holds N float32 samples of a time
                                    series (a dedispersed trial), and the server makes the
                                    spectrum on the GPU as the reference does for a .dat
                                    input (jerk_spectrum_from_timeseries); numbins is taken
                                    as N / 2.  N: a length jerk_realfft takes */
    const double *bird_lobins;   /* time-series requests: birdies to zap after the      */
    const double *bird_hibins;   /* preparation (jerk_zap_birdies; host arrays of        */
    int numbirds;                /* numbirds, valid until the result is polled), as a    */
                                 /* -zaplist run zaps them; 0 = none                     */
} jerk_request;

typedef struct jerk_result {
    long long tag;
    int status;                  /* JERK_OK or the error of this request */
    jerk_cand *cands;            /* free with jerk_free */
    long long ncands;
    double t_submit, t_start, t_done;  /* seconds on a steady clock */
} jerk_result;

int jerk_server_create(jerk_server **server, const jerk_server_config *cfg);
int jerk_server_submit(jerk_server *server, const jerk_request *req);
/* Next finished request within timeout_ms: JERK_OK with *out filled, or
 * JERK_TIMEOUT. */
int jerk_server_poll(jerk_server *server, jerk_result *out, int timeout_ms);
/* out[6]: submitted, finished, failed, queued, peak device bytes, budget. */
void jerk_server_stats(jerk_server *server, long long *out);
/* Bytes copied host->device (host spectra and series) and device->host
 * (hit counts and hit lists) for the requests finished so far. */
void jerk_server_transfer_stats(jerk_server *server, long long *h2d, long long *d2h);
/* Finishes every submitted request, then stops; unpolled results are freed. */
void jerk_server_destroy(jerk_server *server);

/* Statistics (host, double precision). */
double jerk_candidate_sigma(double power, int numsum, double numtrials);
double jerk_power_for_sigma(double sigma, int numsum, double numtrials);

/* The host merge of one spectrum searched in pieces (disjoint rstep ranges
 * on several GPUs, or several calls): the raw hits of all pieces (jerk_hits
 * keys and powers, in any order) are sorted by key -- the reference's
 * insertion order -- decoded with the spectrum's geometry (obs and its
 * fundamental, jerk_subharm_sizes entry 0), given their sigma and inserted
 * with the reference's rule.  The list equals the one a single search of the
 * union of the ranges returns.  Host only (no GPU).  Replaces the order-
 * sensitive merge of the reference's GPU path: sort_search_results and
 * insert_to_cands (src/accel_kernels.cu:997-1010, src/accel_utils_cu.c:857-929,
 * src/accelsearch_lib.c:831-878).  *cands is freed with jerk_free. */
int jerk_merge_hits(const jerk_obs *obs, const jerk_subharm *fundamental,
                    const unsigned long long *keys, const float *powers, long long nhits,
                    jerk_cand **cands, long long *ncands);

/* Candidate insertion with the reference's 15-bin rule over a decoded hit
 * sequence; used by jerk_search, exported for tests. */
long long jerk_insert_hits(const jerk_cand *hits, long long nhits, jerk_cand **cands);

void jerk_free(void *p);
const char *jerk_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
