// Jerk-search kernels for sm_100a (FP32 SIMT; the method is spectral, not a
// dense contraction, so there is no tensor-core path).
//
// Per batch of rsteps (one rstep = corr_uselen interbinned fundamental
// bins), three kernels run on one stream:
//
//  1. prep_kernel      one CTA per (rstep, subharmonic): gathers fftlen/2
//                      spectral bins, block-median normalises them exactly as
//                      the reference does, spreads them to interbins, takes
//                      the forward FFT, and writes the rinds lookup table.
//                      (reference: src/accel_utils.c:1107-1210, done there on
//                      the host; src/accel_utils_cu.c:464-588)
//  2. corr_kernel<N>   one CTA per response-kernel row (w, z) of every
//                      subharmonic with fftlen N; the kernel row stays in
//                      registers while the CTA walks all rsteps of the batch:
//                      multiply by conj(kernel), inverse FFT in shared memory,
//                      |.|^2 / fftlen^2 of the numrs good bins straight to the
//                      ffdot volume.  (reference: src/accel_utils.c:1245-1285;
//                      src/accel_kernels.cu:930-988 + cuFFT)
//  3. harmsum_kernel   one thread per fundamental (w, z, r): the stage-0
//                      threshold, then the subharmonic adds in the reference's
//                      order with a threshold after each stage; hits go to a
//                      compact list through warp-aggregated atomics.
//                      (reference: src/accel_utils.c:1356-1377, 1507-1555;
//                      src/accel_kernels.cu:781-862)
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "jerk_fft.cuh"
#include "jerk_kernels.cuh"

namespace jerk {

// ---------------------------------------------------------------------------
// Exact double-precision index arithmetic (no FMA contraction), as the
// reference's host code computes it (src/accel_utils.c:54-97).

__device__ __forceinline__ double calc_required_r_d(double hf, double rfull)
{
    return __dmul_rn(rint(__dmul_rn(__dmul_rn(2.0, rfull), hf)), 0.5);
}

__device__ __forceinline__ int index_from_r_d(double r, double lor)
{
    return __double2int_rz(__dadd_rn(__dmul_rn(__dsub_rn(r, lor), 2.0), 1e-14));
}

// ---------------------------------------------------------------------------
// 1. Data preparation.

constexpr double kLn2 = 0.69314718055994530942;  // log(2.0), correctly rounded

template <int M>
struct NextPow2 {
    static constexpr int value = (M <= 1) ? 1 : 2 * NextPow2<(M + 1) / 2>::value;
};
template <>
struct NextPow2<1> {
    static constexpr int value = 1;
};

// -locpow local power levels (src/corr_routines.c:309-366): the double
// top-hat of weight ((M/2)/NUMLOCPOWAVG, integer division) * 2/M at offsets
// DELTAAVGBINS+1 .. NUMLOCPOWAVG/2+DELTAAVGBINS either side -- the reference
// applies it by FFT correlation, restated as the direct sum -- with the first
// and last kern_half_width bins taking the nearest interior value.
constexpr int kLocAvg = 20;   // NUMLOCPOWAVG (include/presto.h:100)
constexpr int kLocDelta = 5;  // DELTAAVGBINS (include/presto.h:104)

template <int M>
__device__ __forceinline__ float local_power(const float *pw, int i)
{
    constexpr int khw = kLocAvg / 2 + kLocDelta;
    const double w = (double)((M / 2) / kLocAvg) * 2.0 / (double)M;
    const int c = i < khw ? khw : (i >= M - khw ? M - 1 - khw : i);
    double s = 0.0;
#pragma unroll
    for (int d = kLocDelta + 1; d <= khw; d++)
        s = __dadd_rn(s, __dadd_rn((double)pw[c + d], (double)pw[c - d]));
    return __double2float_rn(__dmul_rn(w, s));
}

// Whether prep_impl<N> keeps the FFT twiddles in shared memory beside its
// buffer, data chunk and sort keys (every length up to 7680), or reads them
// from global memory (10240, whose tables alone take 100 KB).
template <int N>
struct PrepTwInSmem {
    static constexpr int M = N / 2;
    static constexpr bool value =
        (size_t)(fft_buf_len<N>() + FftPlan<N>::twsize() + M) * 8 +
            (size_t)NextPow2<M>::value * 4 <= 200 * 1024;
};

template <int N>
__device__ void prep_impl(const SearchDev &P, int b, int s, float *smem)
{
    constexpr int M = N / 2;  // numdata = fftlen / ACCEL_NUMBETWEEN
    constexpr int MP = NextPow2<M>::value;
    constexpr int R0 = FftPlan<N>::R0;
    const SubDev sd = P.subs[s];
    const StepDev st = P.steps[(P.first_rstep + b) * P.nsubs + s];
    constexpr int TWN = FftPlan<N>::twsize();
    float2 *buf = reinterpret_cast<float2 *>(smem);
    // buffer, twiddles, data chunk, sort keys; at the longest fftlen the
    // twiddles stay in global memory (read through L1) to leave room
    constexpr bool kTwS = PrepTwInSmem<N>::value;
    float2 *tws = buf + fft_buf_len<N>();
    float2 *data = tws + (kTwS ? TWN : 0);
    float *keys = reinterpret_cast<float *>(data + M);
    const float2 *tw = kTwS ? tws : P.twiddles + sd.twoff;
    const int tid = threadIdx.x, nt = blockDim.x;

    if constexpr (kTwS) {
        for (int i = tid; i < TWN; i += nt)
            tws[i] = P.twiddles[sd.twoff + i];
    }

    // get_fourier_amplitudes: M bins from lobin, zero outside the file
    const long long lobin = st.rlo - sd.halfwidth;
    for (int i = tid; i < M; i += nt) {
        const long long bi = lobin - P.lobin + i;
        float2 v = make_float2(0.f, 0.f);
        if (bi >= 0 && bi < P.numbins)
            v = P.spec[bi];
        data[i] = v;
        keys[i] = __fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y));
    }
    for (int i = M + tid; i < MP; i += nt)
        keys[i] = INFINITY;
    __syncthreads();

    double norm = 1.0;
    if (P.nph > 0.0f) {
        norm = __ddiv_rn(1.0, __dsqrt_rn((double)P.nph));
    } else if (P.norm_type == 1) {
        // -locpow: a float norm per bin (src/accel_utils.c:1186-1203)
        static_assert(M >= 2 * (kLocAvg / 2 + kLocDelta), "chunk too short for -locpow");
        for (int i = tid; i < M; i += nt) {
            const float nrm = invsqrtf_ref(local_power<M>(keys, i));
            float2 v = data[i];
            v.x = __fmul_rn(v.x, nrm);
            v.y = __fmul_rn(v.y, nrm);
            data[i] = v;
        }
    } else {
        // median(): the order statistic of rank (M-1)/2 (src/median.c);
        // bitonic sort of the powers, padded with +inf
        for (int k = 2; k <= MP; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = tid; i < MP; i += nt) {
                    const int ixj = i ^ j;
                    if (ixj > i) {
                        const float a = keys[i], c = keys[ixj];
                        const bool up = (i & k) == 0;
                        if ((a > c) == up) {
                            keys[i] = c;
                            keys[ixj] = a;
                        }
                    }
                }
                __syncthreads();
            }
        }
        const double med = (double)keys[(M - 1) / 2];
        norm = __ddiv_rn(1.0, __dsqrt_rn(__ddiv_rn(med, kLn2)));
    }
    if (!(P.nph <= 0.0f && P.norm_type == 1)) {
        for (int i = tid; i < M; i += nt) {
            float2 v = data[i];
            v.x = __double2float_rn(__dmul_rn((double)v.x, norm));
            v.y = __double2float_rn(__dmul_rn((double)v.y, norm));
            data[i] = v;
        }
    }
    __syncthreads();

    // spread_no_pad (data at even interbins) + forward FFT (sign -1).  For a
    // power-of-two fftlen the chunk is scaled by 1/fftlen here, exactly (a
    // power of two), so the correlation's |y|^2 already carries the
    // reference's 1/fftlen^2 and needs no multiply; other lengths keep it.
    // The transform of the spread chunk repeats with period N/2; only the
    // first half is stored (the correlation reads it twice).
    float2 *outp = P.prepped + sd.data_off + (long long)b * N;
    auto in = [&](int r) -> float2 {
        const int m = tid + r * (N / R0);
        return (m & 1) ? make_float2(0.f, 0.f) : data[m >> 1];
    };
    auto out = [&](int m, float2 y) {
        if constexpr (IsPow2<N>::value) {
            constexpr float inv = 1.0f / (float)N;
            y.x = __fmul_rn(y.x, inv);
            y.y = __fmul_rn(y.y, inv);
        }
        if (m < N / 2)
            outp[m] = y;
    };
    fft_block<N, -1>(buf, tw, tid, in, out);

    // rinds: fundamental r -> subharmonic r index (src/accel_utils.c:1114-1123)
    if (sd.numharm > 1) {
        uint16_t *rinds = P.rinds + ((long long)b * P.nsubs + s) * P.corr_uselen;
        const double rlo = (double)st.rlo;
        for (int ii = tid; ii < P.corr_uselen; ii += nt) {
            const double rr = __dadd_rn(st.fullrlo, __dmul_rn((double)ii, 0.5));
            const double subr = calc_required_r_d(sd.harm_fract, rr);
            rinds[ii] = (uint16_t)index_from_r_d(subr, rlo);
        }
    }
}

__device__ __forceinline__ void prep_dispatch(const SearchDev &P, int b, int s)
{
    extern __shared__ float smem[];
    switch (P.subs[s].fftlen) {
#define JERK_PREP_CASE(NN)                   \
    case NN:                                 \
        prep_impl<NN>(P, b, s, smem);        \
        break;
        JERK_PREP_CASE(128)
        JERK_PREP_CASE(192)
        JERK_PREP_CASE(256)
        JERK_PREP_CASE(384)
        JERK_PREP_CASE(512)
        JERK_PREP_CASE(768)
        JERK_PREP_CASE(1024)
        JERK_PREP_CASE(1280)
        JERK_PREP_CASE(2048)
        JERK_PREP_CASE(4096)
        JERK_PREP_CASE(5120)
        JERK_PREP_CASE(7680)
        JERK_PREP_CASE(10240)
        JERK_PREP_CASE(15360)
#undef JERK_PREP_CASE
    default:
        break;
    }
}

__global__ void __launch_bounds__(1024) prep_kernel(const __grid_constant__ SearchDev P)
{
    prep_dispatch(P, blockIdx.x, blockIdx.y);
}

// plan i of the wave: index of the plan that owns flat CTA x
__device__ __forceinline__ int group_plan(const GroupLaunch &M, int x)
{
    int i = 0;
    while (i + 1 < M.n && x >= M.cta0[i + 1])
        i++;
    return i;
}

__global__ void __launch_bounds__(1024) prep_group_kernel(const __grid_constant__ GroupLaunch M)
{
    const int i = group_plan(M, blockIdx.x);
    const int local = blockIdx.x - M.cta0[i];
    const int nsubs = M.P[i].nsubs;
    prep_dispatch(M.P[i], local / nsubs, local % nsubs);
}

// ---------------------------------------------------------------------------
// 2. Correlation: one CTA per kernel row, all rsteps of the batch.

// Occupancy target for corr_kernel: enough CTAs per SM that 128-thread CTAs
// give 16 resident warps (registers are capped to fit); CTAs of 384 threads
// or more run one per SM (two would cap them at 64 registers and spill).
template <int N>
struct CorrOcc {
    static constexpr int T = FftPlan<N>::T;
    static constexpr int value = T >= 384 ? 1 : (T >= 256 ? 2 : (T >= 128 ? 4 : 8));
};

// Shared memory of corr_kernel<N>, in float2: the FFT buffer, the twiddle
// tables and (when that still leaves CorrOcc CTAs per SM) a staging row for
// the next rstep's prepared data.
// Lengths whose twiddle tables do not fit beside the buffer (15360: 158 KB of
// tables) read twiddles and kernel rows from global memory (L1/L2) instead of
// shared memory and registers; 960 threads leave 68 registers a thread.
template <int N>
struct CorrBig {
    static constexpr bool value =
        (size_t)(fft_buf_len<N>() + FftPlan<N>::twsize()) * 8 > 200 * 1024;
};

template <int N>
struct CorrSmem {
    static constexpr int kBase =
        (fft_buf_len<N>() + (CorrBig<N>::value ? 0 : FftPlan<N>::twsize()) + 1) & ~1;
    // the staged row is the prepared chunk's first half (see corr_body)
    static constexpr bool kStage = (size_t)(kBase + N / 2) * 8 * CorrOcc<N>::value <= 220 * 1024;
    static constexpr int value = kBase + (kStage ? N / 2 : 0);
};

// Bulk (TMA engine) copy of one data row into shared memory, completed on an
// mbarrier, and the bounded wait for it.
__device__ __forceinline__ unsigned smem_u32(const void *p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void bulk_row_load(void *dst, const void *src, unsigned bytes,
                                              uint64_t *bar)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}

// Waits for phase `parity` of the mbarrier; gives up after a bounded number
// of polls (each try_wait itself suspends for a bounded time) and returns
// false.
__device__ __forceinline__ bool bar_wait(uint64_t *bar, unsigned parity)
{
    for (int it = 0; it < (1 << 16); it++) {
        unsigned done;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done) : "r"(smem_u32(bar)), "r"(parity) : "memory");
        if (done)
            return true;
    }
    return false;
}

// Status bits written by the kernels (read back after each pass).
constexpr unsigned kStatusRind = 1u;     // harmsum: a subharmonic r index left its row
constexpr unsigned kStatusCopy = 2u;     // corr: a data-row copy did not complete

// A wait that must run out: the correlation's bounded wait (bar_wait) on an
// mbarrier whose phase 0 nothing completes (no copy is involved, so nothing
// is left in flight).  It gives up after its poll limit and reports as a
// data-row copy that never completed would.  Launched by plans whose wait
// probe is on (jerk_debug_wait_probe), one thread.
__global__ void wait_probe_kernel(unsigned int *status)
{
    __shared__ uint64_t s_probe;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&s_probe)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (!bar_wait(&s_probe, 0) && status)
        atomicOr(status, kStatusCopy);
}

cudaError_t launch_wait_probe(unsigned int *status, cudaStream_t st)
{
    wait_probe_kernel<<<1, 1, 0, st>>>(status);
    return cudaGetLastError();
}

// One CTA of a wave: kernel row `row` of the fftlen-N group G, rsteps
// [b0, b1) of the batch.  (A plan's own launch, corr_kernel below, is the
// same code reading its arguments straight from the kernel parameters: the
// body, which reaches them through references, measured 6 % slower at
// fftlen 2048 and spills at 1280, where CTAs of 80 threads run 8 per SM.)
template <int N>
__device__ __forceinline__ void corr_body(const SearchDev &P, const RowGroup &G, const int row,
                                          const int b0, const int b1)
{
    constexpr int R0 = FftPlan<N>::R0;
    constexpr int T = FftPlan<N>::T;
    constexpr int TWN = FftPlan<N>::twsize();
    constexpr bool kStage = CorrSmem<N>::kStage;
    constexpr bool kBig = CorrBig<N>::value;
    extern __shared__ __align__(16) float2 sm2[];
    __shared__ uint64_t s_bar;
    float2 *buf = sm2;
    float2 *tws = sm2 + fft_buf_len<N>();
    float2 *dsm = sm2 + CorrSmem<N>::kBase;  // staged data row (kStage)
    const int tid = threadIdx.x;
    int gi = 0;
    while (gi + 1 < G.n && row >= G.rowstart[gi + 1])
        gi++;
    const int s = G.sub[gi];
    const int lrow = row - G.rowstart[gi];
    const SubDev sd = P.subs[s];
    const float2 *D0 = P.prepped + sd.data_off;

    // The prepared chunk is the FFT of data spread to even interbins, which
    // repeats with period N/2 (X[k + N/2] = X[k]); prep_kernel stores its
    // first half only, and element m of the product reads X[m mod N/2].  In
    // the first-stage butterfly of thread tid, input r is element
    // tid + r N/R0, so inputs r and r + R0/2 read the same value.
    static_assert(R0 % 2 == 0 && (N / R0) * (R0 / 2) == N / 2, "half-row reads");
    constexpr unsigned kRowBytes = N / 2 * sizeof(float2);
    if constexpr (kStage) {
        if (tid == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&s_bar)) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
        if (tid == 0 && b0 < b1)
            bulk_row_load(dsm, D0 + (long long)b0 * N, kRowBytes, &s_bar);
    }

    const float2 *tw = kBig ? P.twiddles + sd.twoff : tws;
    if constexpr (!kBig) {
        for (int i = tid; i < TWN; i += T)
            tws[i] = P.twiddles[sd.twoff + i];
    }


    // the kernel row, in the order this thread's first-stage butterfly reads it
    // (kBig: read from global memory at every rstep instead)
    float2 kreg[R0];
    const float2 *K = P.bank + sd.kern_off + (long long)lrow * N;
    if constexpr (!kBig) {
#pragma unroll
        for (int r = 0; r < R0; r++)
            kreg[r] = K[tid + r * (N / R0)];
    }
    __syncthreads();

    const int offset = sd.halfwidth * 2;  // binoffset * ACCEL_NUMBETWEEN
    const float norm = sd.pownorm;
    for (int b = b0; b < b1; b++) {
        const int numrs = P.steps[(P.first_rstep + b) * P.nsubs + s].numrs;
        float *outp = P.planes + sd.plane_off + (long long)b * sd.plane_size +
                      (long long)lrow * sd.stride;
        // the power is formed for every output and the store predicated on
        // the good-bin range (one unsigned compare): measured faster than a
        // branch around both.  Power-of-two fftlen: 1/fftlen^2 is already in
        // the chunk.
        auto out = [&](int m, float2 y) {
            const int kk = m - offset;
            const float pw = fmaf(y.x, y.x, y.y * y.y);
            const float o = IsPow2<N>::value ? pw : pw * norm;
            if ((unsigned)kk < (unsigned)numrs)
                outp[kk] = o;
        };
        if constexpr (kStage) {
            // rstep b's row is (or will shortly be) in dsm; once every thread
            // has read it, thread 0 starts the copy of rstep b + 1's row
            if (!bar_wait(&s_bar, (b - b0) & 1) && P.status)
                atomicOr(P.status, kStatusCopy);
            auto in = [&](int r) -> float2 {
                // kBig: the kernel row is read from global memory here too
                return cmulconj(dsm[tid + (r % (R0 / 2)) * (N / R0)],
                                kBig ? K[tid + r * (N / R0)] : kreg[r]);
            };
            auto mid = [&] {
                if (tid == 0 && b + 1 < b1) {
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    bulk_row_load(dsm, D0 + (long long)(b + 1) * N, kRowBytes, &s_bar);
                }
            };
            fft_block<N, +1>(buf, tw, tid, in, out, mid);
        } else {
            const float2 *D = D0 + (long long)b * N;
            auto in = [&](int r) -> float2 {
                const int m = tid + r * (N / R0);
                return cmulconj(D[tid + (r % (R0 / 2)) * (N / R0)], kBig ? K[m] : kreg[r]);
            };
            fft_block<N, +1>(buf, tw, tid, in, out);
        }
        __syncthreads();
    }
}

// this CTA's rsteps: all of the batch, or a share of them when a small
// group's rows alone would leave SMs idle (ny > 1 chunks)
__device__ __forceinline__ void rstep_chunk(int nb, int ny, int y, int *b0, int *b1)
{
    const int bchunk = (nb + ny - 1) / ny;
    *b0 = min(nb, y * bchunk);
    *b1 = min(nb, *b0 + bchunk);
}

// A plan's own launch: one CTA per kernel row (blockIdx.x) of the group,
// rsteps of chunk blockIdx.y of gridDim.y.
template <int N>
__global__ void __launch_bounds__(FftPlan<N>::T, CorrOcc<N>::value)
    corr_kernel(const __grid_constant__ SearchDev P, const __grid_constant__ RowGroup G)
{
    constexpr int R0 = FftPlan<N>::R0;
    constexpr int T = FftPlan<N>::T;
    constexpr int TWN = FftPlan<N>::twsize();
    constexpr bool kStage = CorrSmem<N>::kStage;
    constexpr bool kBig = CorrBig<N>::value;
    extern __shared__ __align__(16) float2 sm2[];
    __shared__ uint64_t s_bar;
    float2 *buf = sm2;
    float2 *tws = sm2 + fft_buf_len<N>();
    float2 *dsm = sm2 + CorrSmem<N>::kBase;  // staged data row (kStage)
    const int tid = threadIdx.x;
    const int row = blockIdx.x;
    int gi = 0;
    while (gi + 1 < G.n && row >= G.rowstart[gi + 1])
        gi++;
    const int s = G.sub[gi];
    const int lrow = row - G.rowstart[gi];
    const SubDev sd = P.subs[s];
    const float2 *D0 = P.prepped + sd.data_off;
    // this CTA's rsteps: all of the batch, or a share of them when a small
    // group's rows alone would leave SMs idle (gridDim.y > 1)
    const int bchunk = (P.nb + (int)gridDim.y - 1) / (int)gridDim.y;
    const int b0 = min(P.nb, (int)blockIdx.y * bchunk), b1 = min(P.nb, b0 + bchunk);

    // The prepared chunk is the FFT of data spread to even interbins, which
    // repeats with period N/2 (X[k + N/2] = X[k]); prep_kernel stores its
    // first half only, and element m of the product reads X[m mod N/2].  In
    // the first-stage butterfly of thread tid, input r is element
    // tid + r N/R0, so inputs r and r + R0/2 read the same value.
    static_assert(R0 % 2 == 0 && (N / R0) * (R0 / 2) == N / 2, "half-row reads");
    constexpr unsigned kRowBytes = N / 2 * sizeof(float2);
    if constexpr (kStage) {
        if (tid == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&s_bar)) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
        if (tid == 0 && b0 < b1)
            bulk_row_load(dsm, D0 + (long long)b0 * N, kRowBytes, &s_bar);
    }

    const float2 *tw = kBig ? P.twiddles + sd.twoff : tws;
    if constexpr (!kBig) {
        for (int i = tid; i < TWN; i += T)
            tws[i] = P.twiddles[sd.twoff + i];
    }


    // the kernel row, in the order this thread's first-stage butterfly reads it
    // (kBig: read from global memory at every rstep instead)
    float2 kreg[R0];
    const float2 *K = P.bank + sd.kern_off + (long long)lrow * N;
    if constexpr (!kBig) {
#pragma unroll
        for (int r = 0; r < R0; r++)
            kreg[r] = K[tid + r * (N / R0)];
    }
    __syncthreads();

    const int offset = sd.halfwidth * 2;  // binoffset * ACCEL_NUMBETWEEN
    const float norm = sd.pownorm;
    for (int b = b0; b < b1; b++) {
        const int numrs = P.steps[(P.first_rstep + b) * P.nsubs + s].numrs;
        float *outp = P.planes + sd.plane_off + (long long)b * sd.plane_size +
                      (long long)lrow * sd.stride;
        // the power is formed for every output and the store predicated on
        // the good-bin range (one unsigned compare): measured faster than a
        // branch around both.  Power-of-two fftlen: 1/fftlen^2 is already in
        // the chunk.
        auto out = [&](int m, float2 y) {
            const int kk = m - offset;
            const float pw = fmaf(y.x, y.x, y.y * y.y);
            const float o = IsPow2<N>::value ? pw : pw * norm;
            if ((unsigned)kk < (unsigned)numrs)
                outp[kk] = o;
        };
        if constexpr (kStage) {
            // rstep b's row is (or will shortly be) in dsm; once every thread
            // has read it, thread 0 starts the copy of rstep b + 1's row
            if (!bar_wait(&s_bar, (b - b0) & 1) && P.status)
                atomicOr(P.status, kStatusCopy);
            auto in = [&](int r) -> float2 {
                // kBig: the kernel row is read from global memory here too
                return cmulconj(dsm[tid + (r % (R0 / 2)) * (N / R0)],
                                kBig ? K[tid + r * (N / R0)] : kreg[r]);
            };
            auto mid = [&] {
                if (tid == 0 && b + 1 < b1) {
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    bulk_row_load(dsm, D0 + (long long)(b + 1) * N, kRowBytes, &s_bar);
                }
            };
            fft_block<N, +1>(buf, tw, tid, in, out, mid);
        } else {
            const float2 *D = D0 + (long long)b * N;
            auto in = [&](int r) -> float2 {
                const int m = tid + r * (N / R0);
                return cmulconj(D[tid + (r % (R0 / 2)) * (N / R0)], kBig ? K[m] : kreg[r]);
            };
            fft_block<N, +1>(buf, tw, tid, in, out);
        }
        __syncthreads();
    }
}

// A wave's CTAs reach their plan's arguments by index, which costs registers:
// at fftlen 1280 (80-thread CTAs, 8 per SM, 80 registers) the body spills,
// so those run 5 per SM.
template <int N>
struct CorrGroupOcc {
    static constexpr int value = N == 1280 ? 5 : CorrOcc<N>::value;
};

template <int N>
__global__ void __launch_bounds__(FftPlan<N>::T, CorrGroupOcc<N>::value)
    corr_group_kernel(const __grid_constant__ GroupLaunch M)
{
    const int i = group_plan(M, blockIdx.x);
    const int local = blockIdx.x - M.cta0[i];
    const int ny = M.ny[i];
    int b0, b1;
    rstep_chunk(M.P[i].nb, ny, local % ny, &b0, &b1);
    corr_body<N>(M.P[i], M.G[i], local / ny, b0, b1);
}

// ---------------------------------------------------------------------------
// 2b. Correlation at fftlen 2048 and 1280 on folded kernel rows.
//
// The prepared chunk D repeats with period N/2 (it is the transform of data
// spread to even interbins), so the inverse transform of D conj(K) splits
// into two half-length transforms, one per output parity:
//   y[2m]     = IFFT_{N/2}(D A)[m],  A[k] = conj K[k] + conj K[k + N/2]
//   y[2m + 1] = IFFT_{N/2}(D B)[m],  B[k] = (conj K[k] - conj K[k + N/2]) e^{+2 pi i k/N}
// for k < N/2.  A and B depend only on the kernel row, so a plan folds its
// rows of a folded length once (fold_rows_kernel, in double, each value
// rounded once) and the correlation runs two half-length transforms that read
// each data value once for both: the first radix-2 layer of the full
// transform (its butterflies and twiddles) is gone, and the two transforms
// share every twiddle and every data value.
//
// The half-length plan is [8, 16, R2] for T = N/16 threads (H = N/2 = 128
// R2: 1024 = [8, 16, 8] on 128 threads, 640 = [8, 16, 5] on 80).  Stages 0
// and 2 run the two transforms in the two lanes of packed FP32 instructions
// (Cp, pdft8, pdft5): every butterfly of the even transform has its twin in
// the odd one at the same position with the same twiddle and data value, so
// each instruction does both.  Stage 0 (radix 8, T butterflies): thread j
// does butterfly j of both from the same 8 data values, and applies stage 1's
// input twiddles.  Stage 1 (radix 16, T/2 butterflies per transform): one
// transform per thread in scalar FP32, the first half of the threads the even
// one and the second half the odd one, so every warp works (a scalar
// instruction holds the FP32 pipe for one cycle, a packed one for two: the
// pipe time is the same either way).  Stage 2 (radix R2, 128 butterflies,
// Ns = 128): butterfly j of both, and the lane pair of powers (outputs 2 m,
// 2 m + 1) is one 8-byte store.

static int sm_count();

template <int N>
struct FoldPlan;
// CTAs per SM: 5 at 2048 (93 registers, 44 KB of shared memory); 6 at 1280
template <>
struct FoldPlan<2048> {
    static constexpr int R2 = 8, Occ = 5;
};
template <>
struct FoldPlan<1280> {
    static constexpr int R2 = 5, Occ = 6;
};
template <int N>
struct Fold : FoldPlan<N> {
    static constexpr int H = N / 2;
    static constexpr int T = H / 8;                   // threads, stage-0 butterflies
    static constexpr int Plane = fft_buf_len<H>();     // float2 per transform buffer
    static constexpr int Tw2 = 128 * FoldPlan<N>::R2;  // stage 2: W_H^(r k) at [r 128 + k]
    // shared memory: four transform buffers, stage 0's table, the data row
    static constexpr int Smem = (4 * Plane + 128 + H) * 8;
    static_assert(H == 128 * FoldPlan<N>::R2 && T % 16 == 0, "[8, 16, R2] on N/16 threads");
    static_assert((4 * Plane + 128) % 2 == 0, "16-byte aligned staging row");
};
constexpr int kFoldTw1 = 8 * 16;  // stage 1's roots W_128^(r k) at [r 8 + k] (both lengths)

bool fold_length(int N) { return N == 2048 || N == 1280; }
int fold_occ(int N) { return N == 2048 ? Fold<2048>::Occ : N == 1280 ? Fold<1280>::Occ : 0; }

int fold_twiddle_size(int N)
{
    return N == 2048 ? kFoldTw1 + Fold<2048>::Tw2 : N == 1280 ? kFoldTw1 + Fold<1280>::Tw2 : 0;
}

// Host: the two tables of a folded length, forward sign, in double rounded
// to float.
void fold_twiddle_table(int N, float2 *out)
{
    const double tau = 2.0 * 3.14159265358979323846264338327950288;
    const int H = N / 2, R2 = H / 128;
    for (int r = 0; r < 16; r++)
        for (int k = 0; k < 8; k++) {
            const double a = -tau * (double)(r * k) / 128.0;
            out[r * 8 + k] = make_float2((float)cos(a), (float)sin(a));
        }
    for (int r = 0; r < R2; r++)
        for (int k = 0; k < 128; k++) {
            const double a = -tau * (double)(r * k) / (double)H;
            out[kFoldTw1 + r * 128 + k] = make_float2((float)cos(a), (float)sin(a));
        }
}

// Folded rows: row i of the launch's groups (consecutive over its
// subharmonics) from bank row src[i]; out[i] = A (first half), B (second).
template <int N>
__global__ void fold_rows_kernel(const float2 *__restrict__ bank, const long long *src,
                                 float2 *__restrict__ out, int nrows)
{
    constexpr int H = N / 2;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long row = t / H;
    const int k = (int)(t % H);
    if (row >= nrows)
        return;
    const float2 *K = bank + src[row];
    const float2 k0 = K[k], k1 = K[k + H];
    // conj K[k] +/- conj K[k + N/2], in double
    const double ar = (double)k0.x + (double)k1.x, ai = -(double)k0.y - (double)k1.y;
    const double dr = (double)k0.x - (double)k1.x, di = -(double)k0.y + (double)k1.y;
    double sn, cs;
    sincospi((double)k / (double)H, &sn, &cs);  // e^{+2 pi i k / N}
    float2 *o = out + row * N;
    o[k] = make_float2((float)ar, (float)ai);
    o[k + H] = make_float2((float)(dr * cs - di * sn), (float)(dr * sn + di * cs));
}

cudaError_t launch_fold_rows(int N, const float2 *bank, const long long *src, float2 *out,
                             int nrows, cudaStream_t st)
{
    const long long n = (long long)nrows * (N / 2);
    const unsigned blocks = (unsigned)((n + 255) / 256);
    if (N == 2048)
        fold_rows_kernel<2048><<<blocks, 256, 0, st>>>(bank, src, out, nrows);
    else if (N == 1280)
        fold_rows_kernel<1280><<<blocks, 256, 0, st>>>(bank, src, out, nrows);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

// v (c + i s) with (c, s) the conjugate of a forward table root w: the
// inverse transform's twiddle
__device__ __forceinline__ Cp pmul_conj(const Cp &v, float2 w) { return pmul(v, w.x, -w.y); }

// The rstep loop of one CTA of the folded correlation (both launch forms).
// Shared memory holds four transform buffers (stage 0 writes even / odd,
// stage 1 reads them and writes the other two, stage 2 reads those), each a
// padded float2 plane (pad(), conflict-free for all three stages' access
// patterns), stage 0's table and the staged half data row; stage 2's roots
// are read through L1 (shared by the CTAs of an SM).
// kr[r], ki[r]: the lane pairs (re A, re B), (im A, im B) of the row's
// folded values at k = tid + T r.  steps: the row's subharmonic at b = 0
// (stride nsubs per rstep); out: its volume row at b = 0; norm: the
// subharmonic's 1/fftlen^2, applied to the powers where N is not a power
// of two (prep_kernel scales power-of-two chunks by 1/fftlen instead).
template <int N>
__device__ __forceinline__ void fold_rsteps(float2 *bufE, float2 *bufO, float2 *outE,
                                            float2 *outO, const float2 *tw1,
                                            const float2 *tw2, const float2 *dsm, uint64_t *bar,
                                            const float2 (&kr)[8], const float2 (&ki)[8],
                                            const float2 *D0, const StepDev *steps, int nsubs,
                                            float *out, long long plane_size, int offset,
                                            float norm, int b0, int b1, unsigned *status)
{
    using F = Fold<N>;
    constexpr int T = F::T, H = F::H, R2 = F::R2;
    constexpr int NB1 = T / 2;  // stage-1 butterflies per transform
    constexpr unsigned kRowBytes = H * sizeof(float2);
    const int tid = threadIdx.x;
    for (int b = b0; b < b1; b++) {
        const int numrs = steps[(long long)b * nsubs].numrs;
        float *outp = out + (long long)b * plane_size;
        if (!bar_wait(bar, (b - b0) & 1) && status)
            atomicOr(status, kStatusCopy);
        // stage 0: radix 8 of both transforms from the same data values
        {
            Cp v[8];
#pragma unroll
            for (int r = 0; r < 8; r++) {
                const float2 d = dsm[tid + T * r];
                // d A and d B: (dr ar - di ai, dr ai + di ar) per lane
                v[r].re = fma2(bc(d.x), kr[r], mul2(bc(-d.y), ki[r]));
                v[r].im = fma2(bc(d.x), ki[r], mul2(bc(d.y), kr[r]));
            }
            pdft8(v);
            // stage 1's input twiddles, applied here: element 8 t + r of
            // this stage is input t / (T/16) of stage-1 butterfly
            // (8 t + r) mod (T/2), whose twiddle is W_128^((t / (T/16)) r)
            const float2 *w1 = tw1 + (tid / (T / 16)) * 8;
#pragma unroll
            for (int r = 1; r < 8; r++)
                v[r] = pmul_conj(v[r], w1[r]);
            const int pd = pad(tid * 8);
#pragma unroll
            for (int r = 0; r < 8; r++) {
                bufE[pad_add(pd, r)] = make_float2(v[r].re.x, v[r].im.x);
                bufO[pad_add(pd, r)] = make_float2(v[r].re.y, v[r].im.y);
            }
        }
        __syncthreads();
        // every thread has read the staged row: start the next rstep's copy
        if (tid == 0 && b + 1 < b1) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            bulk_row_load(const_cast<float2 *>(dsm), D0 + (long long)(b + 1) * N, kRowBytes, bar);
        }
        // stage 1: radix 16 (Ns = 8), one transform per thread (scalar): the
        // first T/2 threads butterfly j = tid of the even transform, the rest
        // of the odd one; its input twiddles were applied by stage 0
        {
            const bool odd = tid >= NB1;
            const int j = odd ? tid - NB1 : tid;
            const float2 *src = odd ? bufO : bufE;
            float2 *dst = odd ? outO : outE;
            float2 x[16];
            if constexpr (IsPow2<NB1>::value) {
                const int pj = pad(j);
#pragma unroll
                for (int r = 0; r < 16; r++)
                    x[r] = src[pad_add(pj, r * NB1)];
            } else {
#pragma unroll
                for (int r = 0; r < 16; r++)
                    x[r] = src[pad(j + r * NB1)];
            }
            Dft<16, +1>::run(x);
            const int pq = pad((j >> 3) * 128 + (j & 7));
#pragma unroll
            for (int r = 0; r < 16; r++)
                dst[pad_add(pq, r * 8)] = x[r];
        }
        __syncthreads();
        // stage 2: radix R2 (Ns = 128), butterflies j = tid, tid + T, ... < 128
        // of both
#pragma unroll
        for (int jb = 0; jb < 128; jb += T) {
            const int j = jb + tid;
            if (128 % T == 0 || j < 128) {
                Cp v[R2];
                const int pj = pad(j);
#pragma unroll
                for (int r = 0; r < R2; r++) {
                    const float2 e = outE[pad_add(pj, r * 128)], o = outO[pad_add(pj, r * 128)];
                    v[r].re = make_float2(e.x, o.x);
                    v[r].im = make_float2(e.y, o.y);
                }
#pragma unroll
                for (int r = 1; r < R2; r++)
                    v[r] = pmul_conj(v[r], __ldg(tw2 + r * 128 + j));
                if constexpr (R2 == 8)
                    pdft8(v);
                else
                    pdft5(v);
                // outputs 2 m and 2 m + 1, m = j + 128 r: the lane pair of
                // powers is one 8-byte store (offset and numrs are even)
#pragma unroll
                for (int r = 0; r < R2; r++) {
                    const int kk = 2 * (j + 128 * r) - offset;
                    float2 pw = fma2(v[r].re, v[r].re, mul2(v[r].im, v[r].im));
                    if constexpr (!IsPow2<N>::value)
                        pw = mul2(pw, bc(norm));
                    if ((unsigned)kk < (unsigned)numrs)
                        *reinterpret_cast<float2 *>(outp + kk) = pw;
                }
            }
        }
        // no barrier: the next rstep's stage 0 writes bufE / bufO, last read
        // in stage 1 before the barrier above, and its stage 1 writes outE /
        // outO only after the barrier that follows its stage 0
    }
}

// Set-up shared by both launch forms: carve shared memory, start the first
// data-row copy, stage the twiddles, load this thread's folded values, then
// run the rstep loop.
template <int N>
__device__ __forceinline__ void fold_cta(const SubDev &sd, const float2 *prepped,
                                         const StepDev *steps, int nsubs, float *planes,
                                         int lrow, const float2 *__restrict__ Fr,
                                         const float2 *__restrict__ ftw, int b0, int b1,
                                         unsigned *status)
{
    using F = Fold<N>;
    constexpr int T = F::T, H = F::H;
    extern __shared__ __align__(16) float2 smf[];
    __shared__ uint64_t s_bar;
    float2 *tws = smf + 4 * F::Plane;
    float2 *dsm = tws + kFoldTw1;
    const int tid = threadIdx.x;
    const float2 *D0 = prepped + sd.data_off;
    constexpr unsigned kRowBytes = H * sizeof(float2);

    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&s_bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0 && b0 < b1)
        bulk_row_load(dsm, D0 + (long long)b0 * N, kRowBytes, &s_bar);
    for (int i = tid; i < kFoldTw1; i += T)
        tws[i] = ftw[i];
    float2 kr[8], ki[8];
#pragma unroll
    for (int r = 0; r < 8; r++) {
        const float2 a = Fr[tid + T * r], bb = Fr[H + tid + T * r];
        kr[r] = make_float2(a.x, bb.x);
        ki[r] = make_float2(a.y, bb.y);
    }
    __syncthreads();
    fold_rsteps<N>(smf, smf + F::Plane, smf + 2 * F::Plane, smf + 3 * F::Plane, tws,
                   ftw + kFoldTw1, dsm, &s_bar, kr, ki, D0, steps, nsubs,
                   planes + sd.plane_off + (long long)lrow * sd.stride, sd.plane_size,
                   sd.halfwidth * 2, sd.pownorm, b0, b1, status);
}

// A plan's own launch at a folded length: one CTA per kernel row
// (blockIdx.x) of the group, rsteps of chunk blockIdx.y of gridDim.y; F: the
// group's folded rows in launch order; ftw: the two twiddle tables.
template <int N>
__global__ void __launch_bounds__(Fold<N>::T, Fold<N>::Occ)
    corr_fold_kernel(const __grid_constant__ SearchDev P, const __grid_constant__ RowGroup G,
                     const float2 *__restrict__ F, const float2 *__restrict__ ftw)
{
    const int row = blockIdx.x;
    int gi = 0;
    while (gi + 1 < G.n && row >= G.rowstart[gi + 1])
        gi++;
    const int s = G.sub[gi];
    const int bchunk = (P.nb + (int)gridDim.y - 1) / (int)gridDim.y;
    const int b0 = min(P.nb, (int)blockIdx.y * bchunk), b1 = min(P.nb, b0 + bchunk);
    fold_cta<N>(P.subs[s], P.prepped, P.steps + P.first_rstep * P.nsubs + s, P.nsubs, P.planes,
                row - G.rowstart[gi], F + (long long)row * N, ftw, b0, b1, P.status);
}

template <int N>
__global__ void __launch_bounds__(Fold<N>::T, Fold<N>::Occ)
    corr_fold_group_kernel(const __grid_constant__ GroupLaunch M)
{
    const int i = group_plan(M, blockIdx.x);
    const int local = blockIdx.x - M.cta0[i];
    const int ny = M.ny[i];
    int b0, b1;
    rstep_chunk(M.P[i].nb, ny, local % ny, &b0, &b1);
    const SearchDev &P = M.P[i];
    const RowGroup &G = M.G[i];
    const int row = local / ny;
    int gi = 0;
    while (gi + 1 < G.n && row >= G.rowstart[gi + 1])
        gi++;
    const int s = G.sub[gi];
    fold_cta<N>(P.subs[s], P.prepped, P.steps + P.first_rstep * P.nsubs + s, P.nsubs, P.planes,
                row - G.rowstart[gi], M.fold[i] + (long long)row * N, M.fold_tw[i], b0, b1,
                P.status);
}

template <class K>
static cudaError_t fold_attrs(K kernel, int smem)
{
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared);
    return e;
}

// A wave's plans at a folded length (M.fold, M.fold_tw set).
template <int N>
static cudaError_t launch_corr_fold_group_n(GroupLaunch M, cudaStream_t st)
{
    using F = Fold<N>;
    if (M.n < 1 || M.n > kMaxGroupPlans)
        return cudaErrorInvalidValue;
    cudaError_t e = fold_attrs(corr_fold_group_kernel<N>, F::Smem);
    if (e != cudaSuccess)
        return e;
    const int wave = sm_count() * F::Occ;
    long long total = 0;
    for (int i = 0; i < M.n; i++)
        total += M.G[i].rowstart[M.G[i].n];
    long long x = 0;
    for (int i = 0; i < M.n; i++) {
        const int rows = M.G[i].rowstart[M.G[i].n];
        const int split = total >= 2 * wave ? 1
                          : std::max(1, std::min(M.P[i].nb, (int)((2 * wave + total - 1) / total)));
        M.cta0[i] = (int)x;
        M.ny[i] = split;
        x += (long long)rows * split;
    }
    if (x >= (1ll << 31))
        return cudaErrorInvalidValue;
    M.cta0[M.n] = (int)x;
    corr_fold_group_kernel<N><<<(unsigned)x, F::T, F::Smem, st>>>(M);
    return cudaGetLastError();
}

cudaError_t launch_corr_fold_group(int N, GroupLaunch M, cudaStream_t st)
{
    return N == 2048 ? launch_corr_fold_group_n<2048>(M, st)
           : N == 1280 ? launch_corr_fold_group_n<1280>(M, st)
                       : cudaErrorInvalidValue;
}

template <int N>
static cudaError_t launch_corr_fold_n(const SearchDev &P, const RowGroup &G, int rows,
                                      const float2 *Fr, const float2 *ftw, cudaStream_t st)
{
    using F = Fold<N>;
    cudaError_t e = fold_attrs(corr_fold_kernel<N>, F::Smem);
    if (e != cudaSuccess)
        return e;
    const int wave = sm_count() * F::Occ;
    const int split = rows >= 2 * wave ? 1 : std::max(1, std::min(P.nb, (2 * wave + rows - 1) / rows));
    corr_fold_kernel<N><<<dim3(rows, split), F::T, F::Smem, st>>>(P, G, Fr, ftw);
    return cudaGetLastError();
}

cudaError_t launch_corr_fold(int N, const SearchDev &P, const RowGroup &G, int rows,
                             const float2 *F, const float2 *ftw, cudaStream_t st)
{
    return N == 2048 ? launch_corr_fold_n<2048>(P, G, rows, F, ftw, st)
           : N == 1280 ? launch_corr_fold_n<1280>(P, G, rows, F, ftw, st)
                       : cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------
// 3. Harmonic summing + threshold + compaction.

constexpr int kHarmThreads = 128;

// Append one hit.  Hits are rare (a few per rstep at the usual sigma
// cutoffs), so a plain per-thread atomic costs less than a warp vote on every
// comparison; the host sorts the keys, so their order here does not matter.
__device__ __forceinline__ void record_hit(const SearchDev &P, unsigned long long key, float v)
{
    const unsigned int idx = atomicAdd(P.hit_count, 1u);
    if ((long long)idx < P.max_hits) {
        P.hit_keys[idx] = key;
        P.hit_pows[idx] = v;
    }
}

// Shared memory (dynamic): zrow[s][jj] = zinds_s[jj] * stride_s, the row
// offset inside subharmonic s's volume for fundamental z row jj; rows are
// padded to a multiple of 8 entries (zero offsets past numz0) so a thread's
// 4 or 8 rows load as int4s.
__host__ __device__ __forceinline__ int zrow_pitch(int numz0) { return (numz0 + 7) & ~7; }

size_t harmsum_smem_bytes(int nsubs, int numz0)
{
    return sizeof(int) * (size_t)nsubs * zrow_pitch(numz0);
}

// Thread = one fundamental r (kk) of one w row (ii) of one rstep (b); it
// walks all z rows ZU at a time.  Used where the TMA path's boxes (below)
// do not fit in shared memory.  Per point the float adds run in the
// reference's order: stage 1 adds 1/2, stage 2 adds 1/4 then 3/4, ...
// (src/accel_utils.c:1356-1377 applied stage by stage); after each stage the
// value is compared with that stage's cutoff.  Offsets are 32-bit (the
// batch's volumes hold fewer than 2^32 floats; checked on the host).
template <int S, int ZU>
struct HarmOcc {
    // S <= 5, 4 rows per step: 7 CTAs of 128 threads (72 registers) measured
    // 6 % faster than 6 CTAs (80 registers); 8 CTAs spill
    static constexpr int value = ZU <= 4 ? (S <= 5 ? 7 : 4) : (S <= 5 ? 4 : 2);
};

// L2 prefetch, by the copy engine, of the boxes (HarmTma) that fundamental
// rows [j0, j0 + kPrefetchRows) of this CTA will gather: one tensor prefetch
// per subharmonic, no shared memory, nothing to wait for.
constexpr int kPrefetchRows = 16;

template <int NS>
__device__ __forceinline__ void prefetch_tile(const SearchDev &P, const HarmTma &T, int j0,
                                              const int *rstart, const int *wind, int b)
{
    if (j0 >= P.numz0)
        return;
    for (int s = 0; s < NS; s++) {
        const int zs = s == 0 ? j0 : P.zinds[P.subs[s].zinds_off + j0];
        asm volatile("cp.async.bulk.prefetch.tensor.4d.L2.global.tile [%0, {%1, %2, %3, %4}];"
                     :: "l"(reinterpret_cast<uint64_t>(&T.map[s])), "r"(rstart[s]), "r"(zs),
                        "r"(wind[s]), "r"(b)
                     : "memory");
    }
}

// Rare path of harmsum_kernel: the main loop only collects, per step, which
// (stage, row) pairs crossed their cutoff (bit stage * zu + u of hm); this
// redoes those rows' sums -- the same adds in the same order, so the same
// values -- and records each crossing with the value it had at its stage.
// Offsets are rebuilt here (out of line), so the main loop keeps nothing
// extra live for it: measured 11 % faster than testing and recording inside
// the loop.
template <int S>
__device__ __noinline__ void harmsum_rare_hits(const SearchDev &P, const int *hsm, int pitch,
                                               const unsigned int *s_base, int b, int ii, int kk,
                                               int jj0, unsigned int hm, int zu)
{
    constexpr int NS = 1 << (S - 1);
    const long long rstep = P.first_rstep + b;
    for (int u = 0; u < zu; u++) {
        unsigned int bits = 0;
        for (int st = 0; st < S; st++)
            bits |= ((hm >> (st * zu + u)) & 1u) << st;
        if (!bits)
            continue;
        const int jj = jj0 + u;
        float w = P.planes[s_base[0] + kk + hsm[jj]];
        int s = 1;
        for (int st = 0; st < S; st++) {
            if (st > 0) {
                for (int h = 0; h < (1 << (st - 1)); h++, s++) {
                    unsigned int ri = P.rinds[((long long)b * NS + s) * P.corr_uselen + kk];
                    if (ri >= (unsigned int)P.steps[rstep * NS + s].numrs)
                        ri = 0;  // as the main loop does (and flags)
                    w = __fadd_rn(w, P.planes[s_base[s] + ri + hsm[s * pitch + jj]]);
                }
            }
            if (bits & (1u << st))
                record_hit(P,
                           ((((unsigned long long)rstep * S + st) * P.numw0 + ii) * P.numz0 + jj) *
                                   P.corr_uselen + kk,
                           w);
        }
    }
}

// One CTA: r block bx of fundamental w row ii of rstep b.  T (the tensor maps)
// is read only with PF.
template <int S, int ZU, bool PF>
__device__ __forceinline__ void harmsum_body(const SearchDev &P, const HarmTma *T, const int bx,
                                             const int ii, const int b)
{
    constexpr int kHarmZ = ZU;
    static_assert(ZU == 4 || ZU == 8, "whole int4s of z offsets");
    // the crossing mask hm holds one bit per (stage, row): with more than 32
    // the shifts would be undefined and the compiler may drop whole stages
    static_assert(S * ZU <= 32, "hit mask wider than 32 bits");
    constexpr int NS = 1 << (S - 1);
    extern __shared__ int hsm[];
    __shared__ unsigned int s_base[NS];
    __shared__ int s_numrs[NS];
    const int numz0 = P.numz0;
    const int pitch = zrow_pitch(numz0);
    const int tid = threadIdx.x;
    const int kk = bx * kHarmThreads + tid;
    const bool valid = kk < P.corr_uselen;
    const long long rstep = P.first_rstep + b;

    __shared__ int s_pwind[NS], s_prstart[NS];  // prefetch box corners (PF)
    if (tid < NS) {
        const SubDev sd = P.subs[tid];
        const int wind = tid == 0 ? ii : P.wind[sd.wind_off + ii];
        s_base[tid] = (unsigned int)(sd.plane_off + (long long)b * sd.plane_size +
                                     (long long)wind * sd.numz * sd.stride);
        s_numrs[tid] = P.steps[rstep * NS + tid].numrs;
        if constexpr (PF) {
            const int k0 = bx * kHarmThreads;
            s_pwind[tid] = wind;
            s_prstart[tid] = tid == 0 ? k0
                                      : (int)(P.rinds[((long long)b * NS + tid) * P.corr_uselen + k0] &
                                              ~3u);
        }
    }
    for (int i = tid; i < NS * pitch; i += kHarmThreads) {
        const int s = i / pitch, jj = i - s * pitch;
        const SubDev &sd = P.subs[s];
        int zi = 0;
        if (jj < numz0)
            zi = s == 0 ? jj : P.zinds[sd.zinds_off + jj];
        hsm[i] = zi * sd.stride;
    }
    __syncthreads();

    // per-thread offsets: volume row base + this thread's r index
    unsigned int off[NS];
    off[0] = s_base[0] + (valid ? kk : 0);
#pragma unroll
    for (int s = 1; s < NS; s++) {
        unsigned int ri = valid ? P.rinds[((long long)b * NS + s) * P.corr_uselen + kk] : 0u;
        if (ri >= (unsigned int)s_numrs[s]) {
            // cannot happen for tables built as the reference builds them;
            // record it and read a cell that exists
            atomicOr(P.status, kStatusRind);
            ri = 0;
        }
        off[s] = s_base[s] + ri;
    }
    float cut[S];
#pragma unroll
    for (int st = 0; st < S; st++)
        cut[st] = P.powcut[st];

    const float *planes = P.planes;
    // subharmonics [0, NA) belong to stages 0 .. S-2, [NA, NS) to the last
    constexpr int NA = NS > 1 ? NS / 2 : 1;
    if constexpr (PF) {
        if (tid == 0) {
            prefetch_tile<NS>(P, *T, 0, s_prstart, s_pwind, b);
            prefetch_tile<NS>(P, *T, kPrefetchRows, s_prstart, s_pwind, b);
        }
    }
    for (int jj0 = 0; jj0 < numz0; jj0 += kHarmZ) {
        const bool full = jj0 + kHarmZ <= numz0;
        if constexpr (PF) {
            // one tile ahead of the rows being gathered
            if (tid == 0 && jj0 > 0 && jj0 % kPrefetchRows == 0)
                prefetch_tile<NS>(P, *T, jj0 + kPrefetchRows, s_prstart, s_pwind, b);
        }
        float v[kHarmZ];
        unsigned int hm = 0;  // bit stage * ZU + u: row u crossed that stage's cutoff
        // phase 1: every gather of stages 0 .. S-2 for the four rows in flight
        // at once, then the adds in the reference's order
        {
            float x[NA][kHarmZ];
#pragma unroll
            for (int s = 0; s < NA; s++) {
#pragma unroll
                for (int q = 0; q < kHarmZ / 4; q++) {
                    const int4 z = *reinterpret_cast<const int4 *>(hsm + s * pitch + jj0 + 4 * q);
                    x[s][4 * q + 0] = planes[off[s] + z.x];
                    x[s][4 * q + 1] = planes[off[s] + z.y];
                    x[s][4 * q + 2] = planes[off[s] + z.z];
                    x[s][4 * q + 3] = planes[off[s] + z.w];
                }
            }
#pragma unroll
            for (int u = 0; u < kHarmZ; u++)
                v[u] = x[0][u];
            int s = 1;
#pragma unroll
            for (int stage = 0; stage < (S > 1 ? S - 1 : 1); stage++) {
                if (stage > 0) {
#pragma unroll
                    for (int h = 0; h < (1 << (stage - 1)); h++, s++) {
#pragma unroll
                        for (int u = 0; u < kHarmZ; u++)
                            v[u] = __fadd_rn(v[u], x[s][u]);
                    }
                }
#pragma unroll
                for (int u = 0; u < kHarmZ; u++)
                    hm |= v[u] > cut[stage] ? 1u << (stage * kHarmZ + u) : 0u;
            }
        }
        // phase 2: the last stage's subharmonics
        if constexpr (S > 1) {
            float x[NS - NA][kHarmZ];
#pragma unroll
            for (int s = NA; s < NS; s++) {
#pragma unroll
                for (int q = 0; q < kHarmZ / 4; q++) {
                    const int4 z = *reinterpret_cast<const int4 *>(hsm + s * pitch + jj0 + 4 * q);
                    x[s - NA][4 * q + 0] = planes[off[s] + z.x];
                    x[s - NA][4 * q + 1] = planes[off[s] + z.y];
                    x[s - NA][4 * q + 2] = planes[off[s] + z.z];
                    x[s - NA][4 * q + 3] = planes[off[s] + z.w];
                }
            }
#pragma unroll
            for (int s = NA; s < NS; s++) {
#pragma unroll
                for (int u = 0; u < kHarmZ; u++)
                    v[u] = __fadd_rn(v[u], x[s - NA][u]);
            }
            constexpr int stage = S - 1;
#pragma unroll
            for (int u = 0; u < kHarmZ; u++)
                hm |= v[u] > cut[stage] ? 1u << (stage * kHarmZ + u) : 0u;
        }
        if (!valid)
            hm = 0;
        if (!full) {
            const unsigned int rows = (1u << (numz0 - jj0)) - 1u;
            unsigned int m = 0;
#pragma unroll
            for (int st = 0; st < S; st++)
                m |= rows << (st * kHarmZ);
            hm &= m;
        }
        if (hm)
            harmsum_rare_hits<S>(P, hsm, pitch, s_base, b, ii, kk, jj0, hm, kHarmZ);
    }
}

template <int S, int ZU, bool PF>
__global__ void __launch_bounds__(kHarmThreads, HarmOcc<S, ZU>::value)
    harmsum_kernel(const __grid_constant__ SearchDev P, const __grid_constant__ HarmTma T)
{
    harmsum_body<S, ZU, PF>(P, &T, blockIdx.x, blockIdx.y, blockIdx.z);
}

// The gather form over a wave of plans with S stages each (no prefetch).
template <int S>
__global__ void __launch_bounds__(kHarmThreads, HarmOcc<S, 4>::value)
    harmsum_group_kernel(const __grid_constant__ GroupLaunch M)
{
    const int i = group_plan(M, blockIdx.x);
    const int local = blockIdx.x - M.cta0[i];
    const int nx = M.ny[i], nw = M.P[i].numw0;
    harmsum_body<S, 4, false>(M.P[i], nullptr, local % nx, (local / nx) % nw, local / (nx * nw));
}

// ---------------------------------------------------------------------------
// 3b. Harmonic summing fed by TMA (the default where its boxes fit).
//
// Same thread mapping, same float adds in the same order and the same hit
// keys as harmsum_kernel, so the results are bitwise the same; the
// difference is where the operands come from.  The CTA walks the fundamental
// z rows in tiles of ZT.  For each tile, one thread issues one tensor copy per
// subharmonic (cp.async.bulk.tensor.4d): the box of that subharmonic's
// volume that the tile's 128 fundamental r x ZT fundamental z can touch --
// rows zinds_s[z0] .. + Z[s], cells from the tile's first r index (rounded
// down to 4, the 16-byte rule of the x coordinate) .. + W[s] -- into shared
// memory, completing on an mbarrier.  The threads then gather from shared
// memory, so the global-memory latency that bounds harmsum_kernel is paid by
// the copy engine, many tiles in flight per SM.

template <int S, int ZT>
struct HarmTmaOcc {
    static constexpr int value = S <= 5 ? (ZT <= 8 ? 5 : 3) : (ZT <= 8 ? 3 : 2);
};

template <int S, int ZT>
__global__ void __launch_bounds__(kHarmThreads, HarmTmaOcc<S, ZT>::value)
    harmsum_tma_kernel(const SearchDev P, const __grid_constant__ HarmTma T)
{
    constexpr int NS = 1 << (S - 1);
    constexpr int NA = NS > 1 ? NS / 2 : 1;
    constexpr int ZU = 4;  // z rows per compute step
    static_assert(ZT % ZU == 0, "tile of whole steps");
    extern __shared__ __align__(128) float tsm[];
    // tensor-copy destinations 128-byte aligned whatever the static shared
    // variables before the dynamic block (128 bytes of slack are allocated)
    float *box = tsm + ((128u - (smem_u32(tsm) & 127u)) & 127u) / 4u;
    int *zoff = reinterpret_cast<int *>(box + T.box_floats);  // [NS][pitch]
    __shared__ uint64_t s_bar;
    __shared__ int s_wind[NS], s_rstart[NS], s_numrs[NS];
    const int numz0 = P.numz0;
    const int pitch = zrow_pitch(numz0);
    const int b = blockIdx.z;
    const int ii = blockIdx.y;
    const int tid = threadIdx.x;
    const int k0 = blockIdx.x * kHarmThreads;
    const int kk = k0 + tid;
    const bool valid = kk < P.corr_uselen;
    const long long rstep = P.first_rstep + b;

    if (tid < NS) {
        const SubDev sd = P.subs[tid];
        s_wind[tid] = tid == 0 ? ii : P.wind[sd.wind_off + ii];
        s_rstart[tid] = tid == 0 ? k0
                                 : (int)(P.rinds[((long long)b * NS + tid) * P.corr_uselen + k0] & ~3u);
        s_numrs[tid] = P.steps[rstep * NS + tid].numrs;
    }
    // zoff[s][jj]: offset in the shared buffer of subharmonic s's row for
    // fundamental row jj, within the box of jj's tile
    for (int i = tid; i < NS * pitch; i += kHarmThreads) {
        const int s = i / pitch, jj = i - s * pitch;
        int o = T.boxoff[s];
        if (jj < numz0) {
            const int j0 = jj - jj % ZT;
            const int zi = s == 0 ? jj : P.zinds[P.subs[s].zinds_off + jj];
            const int z0 = s == 0 ? j0 : P.zinds[P.subs[s].zinds_off + j0];
            int dz = zi - z0;
            if (dz < 0 || dz >= T.Z[s]) {  // cannot happen for tables built as the reference builds them
                atomicOr(P.status, kStatusRind);
                dz = 0;
            }
            o += dz * T.W[s];
        }
        zoff[i] = o;
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&s_bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (smem_u32(box) & 127u) {  // unreachable by construction; never issue a misaligned copy
        if (tid == 0)
            atomicOr(P.status, kStatusCopy);
        return;
    }

    // this thread's cell in every box
    int col[NS];
    col[0] = tid;
#pragma unroll
    for (int s = 1; s < NS; s++) {
        int c = 0;
        if (valid) {
            const unsigned int ri = P.rinds[((long long)b * NS + s) * P.corr_uselen + kk];
            c = (int)ri - s_rstart[s];
            if (ri >= (unsigned int)s_numrs[s] || c < 0 || c >= T.W[s]) {
                atomicOr(P.status, kStatusRind);
                c = 0;
            }
        }
        col[s] = c;
    }
    float cut[S];
#pragma unroll
    for (int st = 0; st < S; st++)
        cut[st] = P.powcut[st];

    const int ntiles = (numz0 + ZT - 1) / ZT;
    for (int t = 0; t < ntiles; t++) {
        const int z0 = t * ZT;
        if (tid == 0) {
            // the previous tile's reads (generic proxy) are ordered before
            // this tile's writes by the copy engine (async proxy)
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                         :: "r"(smem_u32(&s_bar)), "r"(T.box_bytes) : "memory");
            for (int s = 0; s < NS; s++) {
                const int zs = s == 0 ? z0 : P.zinds[P.subs[s].zinds_off + z0];
                asm volatile(
                    "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                    " [%0], [%1, {%2, %3, %4, %5}], [%6];"
                    :: "r"(smem_u32(box + T.boxoff[s])), "l"(reinterpret_cast<uint64_t>(&T.map[s])),
                       "r"(s_rstart[s]), "r"(zs), "r"(s_wind[s]), "r"(b), "r"(smem_u32(&s_bar))
                    : "memory");
            }
        }
        const bool ok = bar_wait(&s_bar, t & 1);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicOr(P.status, kStatusCopy);
                bar_wait(&s_bar, t & 1);  // once more, bounded, for the copies in flight
            }
            return;
        }
        const int nrows = min(ZT, numz0 - z0);
        for (int u0 = 0; u0 < nrows; u0 += ZU) {
            const int jj0 = z0 + u0;
            const bool full = u0 + ZU <= nrows;
            float v[ZU];
            {
                float x[NA][ZU];
#pragma unroll
                for (int s = 0; s < NA; s++) {
                    const int4 z = *reinterpret_cast<const int4 *>(zoff + s * pitch + jj0);
                    x[s][0] = box[z.x + col[s]];
                    x[s][1] = box[z.y + col[s]];
                    x[s][2] = box[z.z + col[s]];
                    x[s][3] = box[z.w + col[s]];
                }
#pragma unroll
                for (int u = 0; u < ZU; u++)
                    v[u] = x[0][u];
                int s = 1;
#pragma unroll
                for (int stage = 0; stage < (S > 1 ? S - 1 : 1); stage++) {
                    if (stage > 0) {
#pragma unroll
                        for (int h = 0; h < (1 << (stage - 1)); h++, s++) {
#pragma unroll
                            for (int u = 0; u < ZU; u++)
                                v[u] = __fadd_rn(v[u], x[s][u]);
                        }
                    }
#pragma unroll
                    for (int u = 0; u < ZU; u++) {
                        if (valid && (full || u0 + u < nrows) && v[u] > cut[stage])
                            record_hit(P,
                                       ((((unsigned long long)rstep * S + stage) * P.numw0 + ii) *
                                            numz0 + (jj0 + u)) * P.corr_uselen + kk,
                                       v[u]);
                    }
                }
            }
            if constexpr (S > 1) {
                float x[NS - NA][ZU];
#pragma unroll
                for (int s = NA; s < NS; s++) {
                    const int4 z = *reinterpret_cast<const int4 *>(zoff + s * pitch + jj0);
                    x[s - NA][0] = box[z.x + col[s]];
                    x[s - NA][1] = box[z.y + col[s]];
                    x[s - NA][2] = box[z.z + col[s]];
                    x[s - NA][3] = box[z.w + col[s]];
                }
#pragma unroll
                for (int s = NA; s < NS; s++) {
#pragma unroll
                    for (int u = 0; u < ZU; u++)
                        v[u] = __fadd_rn(v[u], x[s - NA][u]);
                }
                constexpr int stage = S - 1;
#pragma unroll
                for (int u = 0; u < ZU; u++) {
                    if (valid && (full || u0 + u < nrows) && v[u] > cut[stage])
                        record_hit(P,
                                   ((((unsigned long long)rstep * S + stage) * P.numw0 + ii) *
                                        numz0 + (jj0 + u)) * P.corr_uselen + kk,
                                   v[u]);
                }
            }
        }
        __syncthreads();  // every read of this tile's boxes is done
    }
}

// ---------------------------------------------------------------------------
// Launchers (host side of this translation unit).

template <int N>
static size_t prep_bytes_n()
{
    constexpr int M = N / 2;
    constexpr int TW = PrepTwInSmem<N>::value ? FftPlan<N>::twsize() : 0;
    return sizeof(float2) * (size_t)(fft_buf_len<N>() + TW + M) +
           sizeof(float) * (size_t)NextPow2<M>::value;
}

size_t prep_smem_bytes(int maxfft)
{
    size_t b = 0;
#define JERK_PB(NN)                                  \
    if (NN <= maxfft && prep_bytes_n<NN>() > b)      \
        b = prep_bytes_n<NN>();
    JERK_PB(128) JERK_PB(192) JERK_PB(256) JERK_PB(384) JERK_PB(512) JERK_PB(768)
    JERK_PB(1024) JERK_PB(1280) JERK_PB(2048) JERK_PB(4096) JERK_PB(5120) JERK_PB(7680) JERK_PB(10240) JERK_PB(15360)
#undef JERK_PB
    return b;
}

// twiddle tables of every supported fftlen's plan (host)
int fft_twiddle_size(int N)
{
    switch (N) {
#define JERK_TS(NN) case NN: return FftPlan<NN>::twsize();
    JERK_TS(128) JERK_TS(192) JERK_TS(256) JERK_TS(384) JERK_TS(512) JERK_TS(768)
    JERK_TS(1024) JERK_TS(1280) JERK_TS(2048) JERK_TS(4096) JERK_TS(5120) JERK_TS(7680) JERK_TS(10240) JERK_TS(15360)
#undef JERK_TS
    default: return -1;
    }
}

void fft_twiddle_table(int N, float2 *out)
{
    switch (N) {
#define JERK_TT(NN) case NN: fft_stage_twiddles<NN>(out); break;
    JERK_TT(128) JERK_TT(192) JERK_TT(256) JERK_TT(384) JERK_TT(512) JERK_TT(768)
    JERK_TT(1024) JERK_TT(1280) JERK_TT(2048) JERK_TT(4096) JERK_TT(5120) JERK_TT(7680) JERK_TT(10240) JERK_TT(15360)
#undef JERK_TT
    default: break;
    }
}

int prep_threads(int maxfft)
{
    // at least the widest FFT plan's thread count, and at least 256
    int t = 256;
#define JERK_PT(NN)                                  \
    if (NN <= maxfft && FftPlan<NN>::T > t)          \
        t = FftPlan<NN>::T;
    JERK_PT(128) JERK_PT(192) JERK_PT(256) JERK_PT(384) JERK_PT(512) JERK_PT(768)
    JERK_PT(1024) JERK_PT(1280) JERK_PT(2048) JERK_PT(4096) JERK_PT(5120) JERK_PT(7680) JERK_PT(10240) JERK_PT(15360)
#undef JERK_PT
    return (t + 31) / 32 * 32;
}

cudaError_t launch_prep(const SearchDev &P, int maxfft, cudaStream_t st)
{
    const size_t smem = prep_smem_bytes(maxfft);
    cudaError_t e = cudaFuncSetAttribute(prep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess)
        return e;
    prep_kernel<<<dim3(P.nb, P.nsubs), prep_threads(maxfft), smem, st>>>(P);
    return cudaGetLastError();
}

// SMs of the current device (queried once; every B200 has 148)
static int sm_count()
{
    static int n = 0;
    if (n <= 0) {
        int dev = 0, v = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && v > 0)
            n = v;
        else
            return 148;
    }
    return n;
}

template <int N>
static cudaError_t launch_corr_n(const SearchDev &P, const RowGroup &G, int rows, cudaStream_t st)
{
    const size_t smem = sizeof(float2) * CorrSmem<N>::value;
    cudaError_t e = cudaFuncSetAttribute(corr_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(corr_kernel<N>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess)
        return e;
    // a group with fewer rows than two waves of CTAs also splits its rsteps
    const int wave = sm_count() * CorrOcc<N>::value;
    const int split = rows >= 2 * wave ? 1 : std::max(1, std::min(P.nb, (2 * wave + rows - 1) / rows));
    corr_kernel<N><<<dim3(rows, split), FftPlan<N>::T, smem, st>>>(P, G);
    return cudaGetLastError();
}

bool fftlen_supported(int n)
{
    switch (n) {
    case 128: case 192: case 256: case 384: case 512: case 768: case 1024: case 1280:
    case 2048: case 4096: case 5120: case 7680: case 10240: case 15360:
        return true;
    default:
        return false;
    }
}

cudaError_t launch_corr(const SearchDev &P, int fftlen, const RowGroup &G, int rows,
                        cudaStream_t st)
{
    switch (fftlen) {
    case 128: return launch_corr_n<128>(P, G, rows, st);
    case 192: return launch_corr_n<192>(P, G, rows, st);
    case 256: return launch_corr_n<256>(P, G, rows, st);
    case 384: return launch_corr_n<384>(P, G, rows, st);
    case 512: return launch_corr_n<512>(P, G, rows, st);
    case 768: return launch_corr_n<768>(P, G, rows, st);
    case 1024: return launch_corr_n<1024>(P, G, rows, st);
    case 1280: return launch_corr_n<1280>(P, G, rows, st);
    case 2048: return launch_corr_n<2048>(P, G, rows, st);
    case 4096: return launch_corr_n<4096>(P, G, rows, st);
    case 5120: return launch_corr_n<5120>(P, G, rows, st);
    case 7680: return launch_corr_n<7680>(P, G, rows, st);
    case 10240: return launch_corr_n<10240>(P, G, rows, st);
    case 15360: return launch_corr_n<15360>(P, G, rows, st);
    default: return cudaErrorInvalidValue;
    }
}

template <int S, bool PF>
static cudaError_t launch_harmsum_s(const SearchDev &P, const HarmTma &T, cudaStream_t st)
{
    const size_t smem = harmsum_smem_bytes(P.nsubs, P.numz0);
    cudaError_t e = cudaFuncSetAttribute(harmsum_kernel<S, 4, PF>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    const dim3 grid((P.corr_uselen + kHarmThreads - 1) / kHarmThreads, P.numw0, P.nb);
    harmsum_kernel<S, 4, PF><<<grid, kHarmThreads, smem, st>>>(P, T);
    return cudaGetLastError();
}

template <bool PF>
static cudaError_t launch_harmsum_p(const SearchDev &P, const HarmTma &T, cudaStream_t st)
{
    switch (P.nstages) {
    case 1: return launch_harmsum_s<1, PF>(P, T, st);
    case 2: return launch_harmsum_s<2, PF>(P, T, st);
    case 3: return launch_harmsum_s<3, PF>(P, T, st);
    case 4: return launch_harmsum_s<4, PF>(P, T, st);
    case 5: return launch_harmsum_s<5, PF>(P, T, st);
    case 6: return launch_harmsum_s<6, PF>(P, T, st);
    default: return cudaErrorInvalidValue;
    }
}

// The gather kernel; with prefetch, T holds tensor maps whose boxes were
// sized for tiles of kPrefetchRows rows.
cudaError_t launch_harmsum(const SearchDev &P, const HarmTma &T, bool prefetch, cudaStream_t st)
{
    return prefetch ? launch_harmsum_p<true>(P, T, st) : launch_harmsum_p<false>(P, T, st);
}

// ---------------------------------------------------------------------------
// Waves: one launch per kernel kind over the current batches of several
// plans.  The caller fills M.n, M.P and (corr) M.G; the launchers fill the
// CTA ranges.

cudaError_t launch_prep_group(GroupLaunch M, int maxfft, cudaStream_t st)
{
    if (M.n < 1 || M.n > kMaxGroupPlans)
        return cudaErrorInvalidValue;
    int x = 0;
    for (int i = 0; i < M.n; i++) {
        M.cta0[i] = x;
        M.ny[i] = 1;
        x += M.P[i].nb * M.P[i].nsubs;
    }
    M.cta0[M.n] = x;
    const size_t smem = prep_smem_bytes(maxfft);
    cudaError_t e = cudaFuncSetAttribute(prep_group_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    prep_group_kernel<<<x, prep_threads(maxfft), smem, st>>>(M);
    return cudaGetLastError();
}

template <int N>
static cudaError_t launch_corr_group_n(GroupLaunch &M, cudaStream_t st)
{
    const size_t smem = sizeof(float2) * CorrSmem<N>::value;
    cudaError_t e = cudaFuncSetAttribute(corr_group_kernel<N>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(corr_group_kernel<N>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess)
        return e;
    // the single-plan rule, applied to the wave's rows together: fewer rows
    // than two waves of CTAs also split their rsteps
    const int wave = sm_count() * CorrGroupOcc<N>::value;
    long long total = 0;
    for (int i = 0; i < M.n; i++)
        total += M.G[i].rowstart[M.G[i].n];
    long long x = 0;
    for (int i = 0; i < M.n; i++) {
        const int rows = M.G[i].rowstart[M.G[i].n];
        const int split = total >= 2 * wave ? 1
                          : std::max(1, std::min(M.P[i].nb, (int)((2 * wave + total - 1) / total)));
        M.cta0[i] = (int)x;
        M.ny[i] = split;
        x += (long long)rows * split;
    }
    if (x >= (1ll << 31))
        return cudaErrorInvalidValue;
    M.cta0[M.n] = (int)x;
    corr_group_kernel<N><<<(unsigned)x, FftPlan<N>::T, smem, st>>>(M);
    return cudaGetLastError();
}

// CTAs of one full wave of the single-plan correlation / harmonic sum
int corr_wave_ctas(int fftlen)
{
    switch (fftlen) {
#define JERK_CW(NN) case NN: return sm_count() * (fold_length(NN) ? fold_occ(NN) : CorrOcc<NN>::value);
    JERK_CW(128) JERK_CW(192) JERK_CW(256) JERK_CW(384) JERK_CW(512) JERK_CW(768)
    JERK_CW(1024) JERK_CW(1280) JERK_CW(2048) JERK_CW(4096) JERK_CW(5120) JERK_CW(7680)
    JERK_CW(10240) JERK_CW(15360)
#undef JERK_CW
    default: return sm_count();
    }
}

int harmsum_wave_ctas(int nstages)
{
    return sm_count() * (nstages <= 5 ? HarmOcc<5, 4>::value : HarmOcc<6, 4>::value);
}

cudaError_t launch_corr_group(GroupLaunch M, int fftlen, cudaStream_t st)
{
    if (M.n < 1 || M.n > kMaxGroupPlans)
        return cudaErrorInvalidValue;
    switch (fftlen) {
#define JERK_CG(NN) case NN: return launch_corr_group_n<NN>(M, st);
    JERK_CG(128) JERK_CG(192) JERK_CG(256) JERK_CG(384) JERK_CG(512) JERK_CG(768)
    JERK_CG(1024) JERK_CG(1280) JERK_CG(2048) JERK_CG(4096) JERK_CG(5120) JERK_CG(7680)
    JERK_CG(10240) JERK_CG(15360)
#undef JERK_CG
    default: return cudaErrorInvalidValue;
    }
}

template <int S>
static cudaError_t launch_harmsum_group_s(GroupLaunch &M, cudaStream_t st)
{
    size_t smem = 0;
    long long x = 0;
    for (int i = 0; i < M.n; i++) {
        const SearchDev &P = M.P[i];
        smem = std::max(smem, harmsum_smem_bytes(P.nsubs, P.numz0));
        M.cta0[i] = (int)x;
        M.ny[i] = (P.corr_uselen + kHarmThreads - 1) / kHarmThreads;
        x += (long long)M.ny[i] * P.numw0 * P.nb;
    }
    if (x >= (1ll << 31))
        return cudaErrorInvalidValue;
    M.cta0[M.n] = (int)x;
    cudaError_t e = cudaFuncSetAttribute(harmsum_group_kernel<S>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    harmsum_group_kernel<S><<<(unsigned)x, kHarmThreads, smem, st>>>(M);
    return cudaGetLastError();
}

// Every plan of M must have nstages stages.
cudaError_t launch_harmsum_group(GroupLaunch M, int nstages, cudaStream_t st)
{
    if (M.n < 1 || M.n > kMaxGroupPlans)
        return cudaErrorInvalidValue;
    switch (nstages) {
    case 1: return launch_harmsum_group_s<1>(M, st);
    case 2: return launch_harmsum_group_s<2>(M, st);
    case 3: return launch_harmsum_group_s<3>(M, st);
    case 4: return launch_harmsum_group_s<4>(M, st);
    case 5: return launch_harmsum_group_s<5>(M, st);
    case 6: return launch_harmsum_group_s<6>(M, st);
    default: return cudaErrorInvalidValue;
    }
}

size_t harmsum_tma_smem_bytes(const HarmTma &T, int nsubs, int numz0)
{
    return 128 + sizeof(float) * (size_t)T.box_floats + harmsum_smem_bytes(nsubs, numz0);
}

template <int S, int ZT>
static cudaError_t launch_harmsum_tma_s(const SearchDev &P, const HarmTma &T, cudaStream_t st)
{
    const size_t smem = harmsum_tma_smem_bytes(T, P.nsubs, P.numz0);
    cudaError_t e = cudaFuncSetAttribute(harmsum_tma_kernel<S, ZT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(harmsum_tma_kernel<S, ZT>,
                                 cudaFuncAttributePreferredSharedMemoryCarveout,
                                 (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess)
        return e;
    const dim3 grid((P.corr_uselen + kHarmThreads - 1) / kHarmThreads, P.numw0, P.nb);
    harmsum_tma_kernel<S, ZT><<<grid, kHarmThreads, smem, st>>>(P, T);
    return cudaGetLastError();
}

template <int ZT>
static cudaError_t launch_harmsum_tma_z(const SearchDev &P, const HarmTma &T, cudaStream_t st)
{
    switch (P.nstages) {
    case 1: return launch_harmsum_tma_s<1, ZT>(P, T, st);
    case 2: return launch_harmsum_tma_s<2, ZT>(P, T, st);
    case 3: return launch_harmsum_tma_s<3, ZT>(P, T, st);
    case 4: return launch_harmsum_tma_s<4, ZT>(P, T, st);
    case 5: return launch_harmsum_tma_s<5, ZT>(P, T, st);
    case 6: return launch_harmsum_tma_s<6, ZT>(P, T, st);
    default: return cudaErrorInvalidValue;
    }
}

// zt: fundamental z rows per tile (8 or 16), as the boxes in T were sized
cudaError_t launch_harmsum_tma(const SearchDev &P, const HarmTma &T, int zt, cudaStream_t st)
{
    return zt == 8 ? launch_harmsum_tma_z<8>(P, T, st) : launch_harmsum_tma_z<16>(P, T, st);
}

}  // namespace jerk

// ---------------------------------------------------------------------------
// Allocation-free entry point.
//
// Some callers cannot allocate device memory at the moment they need a search
// step: a process whose device memory is handed out up front by a pool it
// does not own, a real-time pipeline that forbids allocation after start-up,
// or code running where cudaMalloc would stall or fail.  For them
// jerk_volume_static computes one subharmonic's ffdot volume for one rstep
// (the prep and correlation kernels above) with all of its working memory --
// the subharmonic and rstep descriptors, the FFT twiddles, the prepared
// spectrum chunk and the rinds table -- in one fixed device array,
// g_static_scratch, compiled into this library.  The caller passes only its
// inputs (spectrum, kernel rows) and its output (the volume).
//
// The array is JERK_STATIC_SCRATCH_BYTES (192 KiB) on every GPU that loads
// the library, held until the process exits; it bounds fftlen to 7680 and
// corr_uselen to 16384.  Every call shares it and it keeps the last call's
// contents (each call rewrites all of it that it reads, so nothing needs
// clearing); calls that overlap on the GPU -- two streams, or two host
// threads -- race on it and must be serialised by the caller.  Host code
// cannot use the array's name as a device address, so the first call on each
// device looks the address up with cudaGetSymbolAddress (with that device
// current); make that first call before any stream capture.  After that a
// call only launches kernels on its stream: the descriptors travel as kernel
// parameters and the FFT twiddles are computed on the device, so nothing is
// copied from host memory.

#define JERK_STATIC_SCRATCH_BYTES (192 * 1024)
static __device__ __align__(256) unsigned char g_static_scratch[JERK_STATIC_SCRATCH_BYTES];

#include <cstdio>
#include <mutex>

#include "jerk.h"

namespace jerk {
namespace {

constexpr int kStaticMaxFft = 7680;
constexpr int kStaticMaxUselen = 16384;
// scratch layout (byte offsets)
constexpr size_t kOffSub = 0;
constexpr size_t kOffStep = 256;
constexpr size_t kOffTw = 512;
constexpr size_t kOffData = kOffTw + 81920;                    // twiddles <= 10240 float2
constexpr size_t kOffRinds = kOffData + 8 * (size_t)kStaticMaxFft;
static_assert(kOffRinds + 2 * (size_t)kStaticMaxUselen <= JERK_STATIC_SCRATCH_BYTES,
              "static scratch layout");

std::mutex g_static_mu;
unsigned char *g_static_addr[64];

int static_fail(int code, const char *msg)
{
    char buf[256];
    snprintf(buf, sizeof buf, "jerk_volume_static: %s", msg);
    return set_error(code, buf);
}

// Radices of one FFT plan, passed by value to the set-up kernel.
struct StaticRadices {
    int n;
    int r[kMaxStages];
};

template <int N>
StaticRadices static_radices()
{
    StaticRadices R{};
    R.n = FftPlan<N>::nstages;
    for (int i = 0; i < R.n; i++)
        R.r[i] = FftPlan<N>::radices[i];
    return R;
}

StaticRadices static_radices_of(int N)
{
    switch (N) {
#define JERK_SR(NN) case NN: return static_radices<NN>();
    JERK_SR(128) JERK_SR(192) JERK_SR(256) JERK_SR(384) JERK_SR(512) JERK_SR(768)
    JERK_SR(1024) JERK_SR(1280) JERK_SR(2048) JERK_SR(4096) JERK_SR(5120) JERK_SR(7680)
#undef JERK_SR
    default: return StaticRadices{};
    }
}

}  // namespace

// Writes the call's descriptors and the plan's per-stage twiddle tables (the
// layout fft_stage_twiddles writes on the host: stage s >= 1 holds
// W_{Ns R}^(r k) at [r Ns + k]) into the static array.  Twiddles are taken in
// double, as on the host, and rounded to float.
__global__ void static_setup_kernel(SubDev sd, StepDev sp, StaticRadices R, int tws,
                                    SubDev *dsub, StepDev *dstep, float2 *dtw)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        *dsub = sd;
        *dstep = sp;
    }
    if (i >= tws)
        return;
    int off = 0, ns = R.r[0];
    for (int s = 1; s < R.n; s++) {
        const int size = ns * R.r[s];
        if (i < off + size) {
            const int idx = i - off, r = idx / ns, k = idx % ns;
            const double a = -2.0 * 3.14159265358979323846264338327950288 * (double)(r * k) /
                             (double)size;
            double sa, ca;
            sincos(a, &sa, &ca);
            dtw[i] = make_float2((float)ca, (float)sa);
            return;
        }
        off += size;
        ns *= R.r[s];
    }
}

}  // namespace jerk

extern "C" int jerk_volume_static(const void *spectrum, long long numbins, long long lobin,
                                  const jerk_subharm *sub, const void *kernels, double fullrlo,
                                  int corr_uselen, float nph, float *volume, int *numrs_out,
                                  long long *rlo_out, void *stream)
{
    using namespace jerk;
    if (!spectrum || !sub || !kernels || !volume || numbins < 1)
        return static_fail(JERK_EINVAL, "null argument");
    const int N = sub->fftlen;
    const int tws = fft_twiddle_size(N);
    if (N > kStaticMaxFft || tws < 0 || (size_t)tws * sizeof(float2) > kOffData - kOffTw)
        return static_fail(JERK_EINVAL, "fftlen beyond the static scratch (at most 7680, and supported)");
    if (corr_uselen <= 0 || corr_uselen % 2 || corr_uselen > kStaticMaxUselen)
        return static_fail(JERK_EINVAL, "corr_uselen beyond the static scratch (even, at most 16384)");
    if (sub->numharm < 1 || sub->harmnum < 1 || sub->numz < 1 || sub->numw < 1)
        return static_fail(JERK_EINVAL, "bad subharmonic");

    // rstep geometry, as jerk_plan_create computes it (src/accel_utils.c:1107-1141)
    const double hf = (double)sub->harmnum / (double)sub->numharm;
    const int rstep = corr_uselen / 2;
    const double lastr = fullrlo + rstep - 0.5;
    const double drlo = rint(2.0 * fullrlo * hf) * 0.5, drhi = rint(2.0 * lastr * hf) * 0.5;
    int numrs = (int)((ceil(drhi) - floor(drlo)) * 2 + 1e-14) + 1;
    if (sub->numharm == 1 && sub->harmnum == 1)
        numrs = corr_uselen;
    else if (numrs % 2)
        numrs = (numrs / 2 + 1) * 2;
    if (numrs + 2 * sub->halfwidth > N)
        return static_fail(JERK_EINVAL, "fftlen too short for the good bins");

    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return static_fail(JERK_ECUDA, "cudaGetDevice failed");
    if (dev < 0 || dev >= 64)
        return static_fail(JERK_EUNSUPPORTED, "device ordinal above 63");
    unsigned char *base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_static_mu);
        if (!g_static_addr[dev]) {
            void *addr = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&addr, g_static_scratch);
            if (e != cudaSuccess || !addr) {
                char msg[160];
                snprintf(msg, sizeof msg, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
                return static_fail(JERK_ECUDA, msg);
            }
            g_static_addr[dev] = (unsigned char *)addr;
        }
        base = g_static_addr[dev];
    }

    SubDev sd{};
    sd.numharm = sub->numharm;
    sd.harmnum = sub->harmnum;
    sd.harm_fract = hf;
    sd.numz = sub->numz;
    sd.numw = sub->numw;
    sd.fftlen = N;
    sd.halfwidth = sub->halfwidth;
    sd.stride = numrs;
    sd.pownorm = (float)(1.0 / (double)(N * N));
    sd.twoff = 0;
    sd.kern_off = 0;
    sd.plane_off = 0;
    sd.plane_size = (long long)sub->numw * sub->numz * numrs;
    sd.data_off = 0;
    StepDev sp{};
    sp.rlo = (long long)floor(drlo);
    sp.fullrlo = fullrlo;
    sp.numrs = numrs;

    // descriptors and twiddles into the array, by a kernel on the call's
    // stream: no copy from host memory
    static_setup_kernel<<<(tws + 255) / 256 > 0 ? (tws + 255) / 256 : 1, 256, 0, st>>>(
        sd, sp, static_radices_of(N), tws, (SubDev *)(base + kOffSub),
        (StepDev *)(base + kOffStep), (float2 *)(base + kOffTw));
    cudaError_t e = cudaGetLastError();

    SearchDev P{};
    P.spec = (const float2 *)spectrum;
    P.numbins = numbins;
    P.lobin = lobin;
    P.nsubs = 1;
    P.nstages = 1;
    P.corr_uselen = corr_uselen;
    P.numz0 = sub->numz;
    P.numw0 = sub->numw;
    P.norm_type = 0;
    P.nph = nph;
    P.subs = (const SubDev *)(base + kOffSub);
    P.steps = (const StepDev *)(base + kOffStep);
    P.bank = (const float2 *)kernels;
    P.twiddles = (const float2 *)(base + kOffTw);
    P.prepped = (float2 *)(base + kOffData);
    P.planes = volume;
    P.rinds = (uint16_t *)(base + kOffRinds);
    P.first_rstep = 0;
    P.nb = 1;
    if (e == cudaSuccess)
        e = launch_prep(P, N, st);
    if (e == cudaSuccess) {
        RowGroup G{};
        G.n = 1;
        G.sub[0] = 0;
        G.rowstart[0] = 0;
        G.rowstart[1] = sub->numw * sub->numz;
        e = launch_corr(P, N, G, G.rowstart[1], st);
    }
    if (e != cudaSuccess)
        return static_fail(JERK_ECUDA, cudaGetErrorString(e));
    if (numrs_out)
        *numrs_out = numrs;
    if (rlo_out)
        *rlo_out = sp.rlo;
    return JERK_OK;
}
