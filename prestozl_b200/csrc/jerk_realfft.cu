// The spectrum of a time series on the GPU, as the reference prepares a
// ".dat" input before its search (src/accel_utils.c:1696-1753): a forward
// real FFT in PRESTO's packing (realfft, src/fastffts.c:163-235, isign -1)
// followed by red-noise removal (deredden, src/accel_utils.c:1557-1633).
//
// Real FFT of n = 2M samples.  The samples are read as M complex values
// z[m] = x[2m] + i x[2m+1]; their M-point FFT Z is taken in four steps with
// M = R1 * R2 (R1, R2 block-FFT sizes from 128 to 10240: powers of two and
// products with 3 and 5), each step one block-wide FFT per CTA from
// jerk_fft.cuh:
//   1. columns: for each m2 < R2, the R1-point FFT over m1 of z[m2 + R2 m1],
//      times exp(-2 pi i m2 k1 / M), stored as row k1 of an R1 x R2 scratch;
//   2. rows: for each k1 < R1, the R2-point FFT of that row, stored to
//      Z[k1 + R1 k2] in the output;
//   3. in place on the output: X[k] = (Z[k] + conj Z[M-k]) / 2
//      - (i/2) exp(-2 pi i k / n) (Z[k] - conj Z[M-k]), one thread per
//      pair (k, M-k) in double, and X[0] = (DC, Nyquist) packed as the
//      reference packs them.
// No scaling (the reference's forward transform is unnormalised).  The
// FFTs run in FP32 like the reference's, so values agree with the
// reference's to FP32 rounding, not bitwise.
//
// Red-noise removal is bit-exact with the reference.  Its blocks depend only
// on where the walk stops: block 0 is bins [1, 7); each later block starts
// where the previous one ended and is (int)(6 ln(start)) bins long (at most
// 200); a block exists while it ends below numamps.  The host walks this
// sequence once with the C library's log, as the reference does, and keeps it
// as runs of blocks of equal length (about 130 runs cover 2^31 bins), passed
// to the kernels by value.  One warp per block takes the median power (the
// value of rank (n-1)/2, which the reference's quickselect returns) over
// ln 2 (a bitonic sort in registers); one warp per segment between block
// midpoints then scales its bins by
// invsqrtf of the linearly interpolated level, in the reference's float and
// double steps.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <vector>

#include "jerk.h"
#include "jerk_fft.cuh"
#include "jerk_kernels.cuh"

namespace jerk {
namespace {

// R1, R2: the block-FFT sizes from 128 to 10240 (powers of two and the mixed
// sizes with factors 3 and 5 that jerk_fft.cuh plans)
constexpr int kRfSizes[] = {128, 192, 256, 384, 512, 768, 1024, 1280, 2048,
                            4096, 5120, 7680, 8192, 10240};

// ---------------------------------------------------------------------------
// real FFT kernels

// Entry i of the per-stage twiddle tables of FftPlan<N> (the layout
// fft_stage_twiddles writes on the host), computed in double.
template <int N, int S>
__device__ __forceinline__ void stage_twiddle(int i, float2 *tw)
{
    using P = FftPlan<N>;
    if constexpr (S < P::nstages) {
        constexpr int R = P::radices[S];
        constexpr int OFF = P::twoff(S);
        constexpr int NS = (P::twoff(S + 1) - OFF) / R;
        if (i < OFF + NS * R) {
            const int r = (i - OFF) / NS, k = (i - OFF) % NS;
            double s, c;
            sincospi(-2.0 * (double)(r * k) / (double)(NS * R), &s, &c);
            tw[i] = make_float2((float)c, (float)s);
        } else {
            stage_twiddle<N, S + 1>(i, tw);
        }
    }
}

template <int N>
__global__ void rf_twiddle_kernel(float2 *tw)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < FftPlan<N>::twsize())
        stage_twiddle<N, 1>(i, tw);
}

// Step 1: CTA m2 transforms column m2 of z (stride R2) and stores row k1 of
// the scratch at a[k1 * R2 + m2], times exp(-2 pi i m2 k1 / M).  The twiddle
// is the double product of two per-CTA tables, exp(-2 pi i m2 lo / M) and
// exp(-2 pi i m2 64 hi / M) for k1 = 64 hi + lo (exponents reduced mod M
// exactly), rounded once to float.
constexpr int kTwLo = 64;
template <int R1>
__global__ void __launch_bounds__(FftPlan<R1>::T)
    rf_column_kernel(const float2 *__restrict__ z, int R2, const float2 *__restrict__ tw,
                     float2 *__restrict__ a)
{
    constexpr int T = FftPlan<R1>::T;
    constexpr int NHI = (R1 + kTwLo - 1) / kTwLo;
    extern __shared__ float2 rf_buf[];
    __shared__ double2 t_lo[kTwLo], t_hi[NHI];
    const int tid = threadIdx.x;
    const int m2 = blockIdx.x;
    const long long M = (long long)R1 * R2;
    for (int i = tid; i < kTwLo + NHI; i += T) {
        const long long e = i < kTwLo ? ((long long)m2 * i) % M
                                      : ((long long)m2 * kTwLo * (i - kTwLo)) % M;
        double s, c;
        sincospi(-2.0 * (double)e / (double)M, &s, &c);
        if (i < kTwLo)
            t_lo[i] = make_double2(c, s);
        else
            t_hi[i - kTwLo] = make_double2(c, s);
    }
    // fft_block's first barrier orders these writes before the reads in out()
    auto in = [&](int r) -> float2 { return z[m2 + (size_t)R2 * (size_t)(tid + r * T)]; };
    auto out = [&](int k1, float2 y) {
        const double2 u = t_hi[k1 / kTwLo], v = t_lo[k1 % kTwLo];
        const float2 w = make_float2((float)(u.x * v.x - u.y * v.y), (float)(u.x * v.y + u.y * v.x));
        a[(size_t)k1 * R2 + m2] = cmul(y, w);
    };
    fft_block<R1, -1>(rf_buf, tw, tid, in, out);
}

// Step 2: CTA k1 transforms row k1 of the scratch and stores Z[k1 + R1 k2].
template <int R2>
__global__ void __launch_bounds__(FftPlan<R2>::T)
    rf_row_kernel(const float2 *__restrict__ a, int R1, const float2 *__restrict__ tw,
                  float2 *__restrict__ zout)
{
    constexpr int T = FftPlan<R2>::T;
    extern __shared__ float2 rf_buf[];
    const int tid = threadIdx.x;
    const int k1 = blockIdx.x;
    const float2 *row = a + (size_t)k1 * R2;
    auto in = [&](int r) -> float2 { return row[tid + r * T]; };
    auto out = [&](int k2, float2 y) { zout[k1 + (size_t)R1 * k2] = y; };
    fft_block<R2, -1>(rf_buf, tw, tid, in, out);
}

// Step 3, in place: thread k (0 <= k <= M/2) turns Z[k], Z[M-k] into X[k],
// X[M-k].  With h = (Z[k] + conj Z[M-k]) / 2, d = Z[k] - conj Z[M-k] and
// g = W d, W = exp(-i pi k / M):
//   X[k]   = (h.x + g.y / 2,  h.y - g.x / 2)
//   X[M-k] = (h.x - g.y / 2, -h.y - g.x / 2)
__global__ void rf_post_kernel(float2 *x, long long M)
{
    const long long half = M / 2;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k <= half;
         k += (long long)gridDim.x * blockDim.x) {
        if (k == 0) {
            const float2 z0 = x[0];
            x[0] = make_float2(z0.x + z0.y, z0.x - z0.y);
            continue;
        }
        const float2 a = x[k], b = x[M - k];
        const double hx = 0.5 * ((double)a.x + (double)b.x);
        const double hy = 0.5 * ((double)a.y - (double)b.y);
        const double dx = (double)a.x - (double)b.x;
        const double dy = (double)a.y + (double)b.y;
        double s, c;
        sincospi(-(double)k / (double)M, &s, &c);
        const double gx = c * dx - s * dy, gy = c * dy + s * dx;
        x[k] = make_float2((float)(hx + 0.5 * gy), (float)(hy - 0.5 * gx));
        if (k != M - k)
            x[M - k] = make_float2((float)(hx - 0.5 * gy), (float)(-hy - 0.5 * gx));
    }
}

template <int R>
cudaError_t rf_launch_twiddles(float2 *tw, cudaStream_t st)
{
    constexpr int n = FftPlan<R>::twsize();
    rf_twiddle_kernel<R><<<(n + 255) / 256, 256, 0, st>>>(tw);
    return cudaGetLastError();
}

template <int R1>
cudaError_t rf_launch_columns(const float2 *z, int R2, const float2 *tw, float2 *a, cudaStream_t st)
{
    const int smem = (int)(sizeof(float2) * fft_buf_len<R1>());
    cudaError_t e = cudaFuncSetAttribute(rf_column_kernel<R1>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess)
        return e;
    rf_column_kernel<R1><<<R2, FftPlan<R1>::T, smem, st>>>(z, R2, tw, a);
    return cudaGetLastError();
}

template <int R2>
cudaError_t rf_launch_rows(const float2 *a, int R1, const float2 *tw, float2 *zout, cudaStream_t st)
{
    const int smem = (int)(sizeof(float2) * fft_buf_len<R2>());
    cudaError_t e = cudaFuncSetAttribute(rf_row_kernel<R2>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess)
        return e;
    rf_row_kernel<R2><<<R1, FftPlan<R2>::T, smem, st>>>(a, R1, tw, zout);
    return cudaGetLastError();
}

// Runtime dispatch over kRfSizes.
template <template <int> class F, class... A>
cudaError_t rf_dispatch(int R, A... args)
{
    switch (R) {
    case 128: return F<128>::run(args...);
    case 192: return F<192>::run(args...);
    case 256: return F<256>::run(args...);
    case 384: return F<384>::run(args...);
    case 512: return F<512>::run(args...);
    case 768: return F<768>::run(args...);
    case 1024: return F<1024>::run(args...);
    case 1280: return F<1280>::run(args...);
    case 2048: return F<2048>::run(args...);
    case 4096: return F<4096>::run(args...);
    case 5120: return F<5120>::run(args...);
    case 7680: return F<7680>::run(args...);
    case 8192: return F<8192>::run(args...);
    case 10240: return F<10240>::run(args...);
    default: return cudaErrorInvalidValue;
    }
}
template <int R> struct RfTw {
    static cudaError_t run(float2 *tw, cudaStream_t st) { return rf_launch_twiddles<R>(tw, st); }
};
template <int R> struct RfCol {
    static cudaError_t run(const float2 *z, int R2, const float2 *tw, float2 *a, cudaStream_t st)
    {
        return rf_launch_columns<R>(z, R2, tw, a, st);
    }
};
template <int R> struct RfRow {
    static cudaError_t run(const float2 *a, int R1, const float2 *tw, float2 *zo, cudaStream_t st)
    {
        return rf_launch_rows<R>(a, R1, tw, zo, st);
    }
};

template <int R> struct RfTwSize {
    static cudaError_t run(int *out)
    {
        *out = FftPlan<R>::twsize();
        return cudaSuccess;
    }
};

int rf_twsize(int R)
{
    int n = -1;
    return rf_dispatch<RfTwSize>(R, &n) == cudaSuccess ? n : -1;
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// M = n / 2 = R1 * R2 with R1, R2 in kRfSizes, the most balanced pair
// (R1 >= R2); false when n is odd or M has no such factorisation.
bool rf_split(long long n, int *R1, int *R2)
{
    if (n < 2 || (n & 1))
        return false;
    const long long M = n / 2;
    bool found = false;
    for (int a : kRfSizes)
        for (int b : kRfSizes)
            if (a >= b && (long long)a * b == M && (!found || a - b < *R1 - *R2)) {
                *R1 = a;
                *R2 = b;
                found = true;
            }
    return found;
}

// scratch: [M float2 | R1 twiddles | R2 twiddles], each region 256-aligned
size_t rf_scratch(int R1, int R2)
{
    return align256(sizeof(float2) * (size_t)R1 * R2) + align256(sizeof(float2) * rf_twsize(R1)) +
           align256(sizeof(float2) * rf_twsize(R2));
}

// ---------------------------------------------------------------------------
// red-noise removal

constexpr int kDrInit = 6, kDrMax = 200;  // initialbuflen, maxbuflen
constexpr int kDrRuns = 192;

// Blocks first .. first + count - 1 start at start + (b - first) * len.
struct DrRun {
    int first, start, len, count;
};
struct DrRuns {
    int n;
    DrRun r[kDrRuns];
};
static_assert(sizeof(DrRuns) <= 4000, "kernel parameter space");

__device__ __forceinline__ int2 dr_block(const DrRuns &R, int b)
{
    int lo = 0, hi = R.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (R.r[mid].first <= b)
            lo = mid;
        else
            hi = mid - 1;
    }
    const DrRun &u = R.r[lo];
    return make_int2(u.start + (b - u.first) * u.len, u.len);
}

__device__ __forceinline__ float dr_power(float2 v)
{
    return __fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y));
}

constexpr int kDrWarps = 8;

// Ascending bitonic sort of 128 values held 4 per lane (value e = lane + 32 j
// in v[j]) across one warp.
__device__ __forceinline__ void warp_sort128(float (&v)[4], int lane)
{
#pragma unroll
    for (int s = 2; s <= 128; s <<= 1) {
#pragma unroll
        for (int d = s >> 1; d > 0; d >>= 1) {
            if (d >= 32) {
                const int dj = d >> 5;
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    if ((j & dj) == 0) {
                        const bool asc = ((lane + 32 * j) & s) == 0;
                        const float a = v[j], b = v[j | dj];
                        v[j] = asc ? fminf(a, b) : fmaxf(a, b);
                        v[j | dj] = asc ? fmaxf(a, b) : fminf(a, b);
                    }
                }
            } else {
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int e = lane + 32 * j;
                    const float o = __shfl_xor_sync(0xffffffffu, v[j], d);
                    const bool keep_min = (((e & s) == 0) == ((e & d) == 0));
                    v[j] = keep_min ? fminf(v[j], o) : fmaxf(v[j], o);
                }
            }
        }
    }
}

// One warp per block: level[b] = median power / ln 2.  Blocks are at most 128
// bins long below 2^31 bins ((int)(6 ln 2^31) = 128): sorted in registers,
// padded with +inf; the value at sorted position (n-1)/2 is the one the
// reference's quickselect returns.  (Longer blocks, which the walk never
// makes, would take the stable-rank count.)
__global__ void __launch_bounds__(32 * kDrWarps)
    dr_level_kernel(const float2 *__restrict__ x, const __grid_constant__ DrRuns runs, int nb,
                    double ln2, float *__restrict__ level)
{
    __shared__ float pw[kDrWarps][kDrMax];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b = blockIdx.x * kDrWarps + w;
    if (b >= nb)
        return;  // whole warps leave; only warp-level syncs below
    const int2 blk = dr_block(runs, b);
    const int n = blk.y;
    const int k = (n - 1) / 2;
    if (n <= 128) {
        float v[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int i = lane + 32 * j;
            v[j] = i < n ? dr_power(x[blk.x + i]) : INFINITY;
        }
        warp_sort128(v, lane);
        const float m0 = __shfl_sync(0xffffffffu, v[0], k & 31);
        const float m1 = __shfl_sync(0xffffffffu, v[1], k & 31);
        if (lane == 0)
            level[b] = (float)((double)(k < 32 ? m0 : m1) / ln2);
        return;
    }
    float *p = pw[w];
    for (int i = lane; i < n; i += 32)
        p[i] = dr_power(x[blk.x + i]);
    __syncwarp();
    for (int i = lane; i < n; i += 32) {
        const float v = p[i];
        int pos = 0;
        for (int j = 0; j < n; j++) {
            const float u = p[j];
            pos += (u < v) | ((u == v) & (j < i));
        }
        if (pos == k)
            level[b] = (float)((double)v / ln2);
    }
}

// One warp per segment s = 0..nb: segment 0 is bins [1, mid(0)) at the
// constant level[0]; segment s is [mid(s-1), mid(s)) (mid(nb) = numamps)
// running from level[s-1] with the slope toward level[s] (the tail keeps the
// last slope, or 1 when there is one block).  mid(b) = start + len / 2.
// Bin 0 becomes (1, bin0_imag).
__global__ void __launch_bounds__(32 * kDrWarps)
    dr_scale_kernel(float2 *__restrict__ x, const __grid_constant__ DrRuns runs, int nb,
                    int numamps, const float *__restrict__ level, float bin0_imag)
{
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = blockIdx.x * kDrWarps + w;
    if (s > nb)
        return;
    int lo, hi;
    float base, slope = 0.0f;
    const bool flat = s == 0;
    if (flat) {
        const int2 b0 = dr_block(runs, 0);
        lo = 1;
        hi = b0.x + b0.y / 2;
        base = level[0];
        if (lane == 0)
            x[0] = make_float2(1.0f, bin0_imag);
    } else {
        const int2 prev = dr_block(runs, s - 1);
        lo = prev.x + prev.y / 2;
        base = level[s - 1];
        if (s < nb) {
            const int2 cur = dr_block(runs, s);
            hi = cur.x + cur.y / 2;
        } else {
            hi = numamps;
        }
        const int bb = s < nb ? s : nb - 1;
        if (bb >= 1) {
            const int la = dr_block(runs, bb - 1).y, lb = dr_block(runs, bb).y;
            slope = (float)((double)__fsub_rn(level[bb], level[bb - 1]) / (0.5 * (double)(la + lb)));
        } else {
            slope = 1.0f;
        }
    }
    for (int ind = lo + lane; ind < hi; ind += 32) {
        const float lv = flat ? base : __fadd_rn(base, __fmul_rn(slope, (float)(ind - lo)));
        const float nrm = invsqrtf_ref(lv);
        float2 v = x[ind];
        v.x = __fmul_rn(v.x, nrm);
        v.y = __fmul_rn(v.y, nrm);
        x[ind] = v;
    }
}

// The block walk from bin 1, kept as runs of equal length.  Shared by every
// call; extended under the lock as longer spectra arrive.
std::mutex g_dr_mu;
std::vector<DrRun> g_dr_runs;  // complete runs plus the open last one
long long g_dr_next = 0;       // start of the first block not yet walked

int dr_len(long long binnum)
{
    const int l = (int)(kDrInit * std::log((double)binnum));
    return l > kDrMax ? kDrMax : l;
}

// Walk until the next block's start passes limit.
void dr_extend(long long limit)
{
    if (g_dr_runs.empty()) {
        g_dr_runs.push_back({0, 1, kDrInit, 1});
        g_dr_next = 1 + kDrInit;
    }
    while (g_dr_next <= limit) {
        const int len = dr_len(g_dr_next);
        DrRun &last = g_dr_runs.back();
        const int nblk = last.first + last.count;
        if (len == last.len && last.first > 0)
            last.count++;
        else
            g_dr_runs.push_back({nblk, (int)g_dr_next, len, 1});
        g_dr_next += len;
    }
}

// The runs of the blocks of a numamps-bin spectrum: block 0, then every
// block b >= 1 with start + len < numamps.  Returns the block count, or -1.
int dr_layout(int numamps, DrRuns *out)
{
    std::lock_guard<std::mutex> lock(g_dr_mu);
    dr_extend(numamps);
    int nb = 0, nr = 0;
    for (const DrRun &u : g_dr_runs) {
        int take = 0;
        if (u.first == 0) {
            take = 1;
        } else {
            // blocks j < count with start + j len + len < numamps
            const long long room = (long long)numamps - u.start - u.len;  // need j * len < room
            if (room > 0)
                take = (int)std::min<long long>(u.count, (room + u.len - 1) / u.len);
        }
        if (take == 0)
            break;
        if (nr == kDrRuns)
            return -1;
        out->r[nr++] = {u.first, u.start, u.len, take};
        nb = u.first + take;
        if (take < u.count)
            break;
    }
    out->n = nr;
    return nb;
}

size_t dr_scratch(int numamps)
{
    return align256(sizeof(float) * (size_t)(numamps / kDrInit + 2));
}

// ---------------------------------------------------------------------------
// birdie zapping (zapbirds from memory, src/zapping.c:29-81)

constexpr int kZapBins = 200;  // MEDIANBINS (src/zapping.c:3)
constexpr int kZapThreads = 256;

// One birdie.  The median powers (rank 99 of 200) of the bins
// [lobin - 300, lobin - 100) and [hibin - 100, hibin + 100), read before any
// bin is written (bins at or past numamps read as zeros, as the reference's
// zero-padded buffer gives them), set avgamp = sqrt(0.5 (mlo + mhi) / ln 2);
// bins [floor(lobin), ceil(hibin)) become (avgamp, 0).
__global__ void __launch_bounds__(kZapThreads)
    zap_kernel(float2 *__restrict__ x, long long numamps, double lobin, double hibin,
               double neg_log_half)
{
    __shared__ float p[2][kZapBins];
    __shared__ float med[2];
    const int tid = threadIdx.x;
    const long long first[2] = {(long long)(lobin - 3 * kZapBins / 2),
                                (long long)(hibin - kZapBins / 2)};
#pragma unroll
    for (int w = 0; w < 2; w++)
        for (int i = tid; i < kZapBins; i += kZapThreads) {
            const long long b = first[w] + i;
            const float2 v = (b >= 0 && b < numamps) ? x[b] : make_float2(0.f, 0.f);
            p[w][i] = dr_power(v);
        }
    __syncthreads();
    constexpr int k = (kZapBins - 1) / 2;
#pragma unroll
    for (int w = 0; w < 2; w++)
        for (int i = tid; i < kZapBins; i += kZapThreads) {
            const float v = p[w][i];
            int pos = 0;
            for (int j = 0; j < kZapBins; j++) {
                const float u = p[w][j];
                pos += (u < v) | ((u == v) & (j < i));
            }
            if (pos == k)
                med[w] = v;
        }
    __syncthreads();
    const float avgamp =
        (float)__dsqrt_rn(__ddiv_rn(0.5 * (double)__fadd_rn(med[0], med[1]), neg_log_half));
    const long long lo = (long long)floor(lobin), hi = (long long)ceil(hibin);
    for (long long b = lo + tid; b < hi; b += kZapThreads)
        if (b >= 0 && b < numamps)
            x[b] = make_float2(avgamp, 0.f);
}

}  // namespace
}  // namespace jerk

using namespace jerk;

extern "C" long long jerk_realfft_scratch_bytes(long long n)
{
    int R1, R2;
    if (!rf_split(n, &R1, &R2))
        return 0;
    return (long long)rf_scratch(R1, R2);
}

extern "C" int jerk_realfft(const float *timeseries, long long n, void *spectrum, void *scratch,
                            long long scratch_bytes, void *stream)
{
    int R1, R2;
    if (!rf_split(n, &R1, &R2))
        return set_error(JERK_EUNSUPPORTED,
                         "jerk_realfft: n must be 2 R1 R2 with R1, R2 in {128, 192, 256, 384, "
                         "512, 768, 1024, 1280, 2048, 4096, 5120, 7680, 8192, 10240}");
    if (!timeseries || !spectrum || !scratch)
        return set_error(JERK_EINVAL, "jerk_realfft: null pointer");
    if (((uintptr_t)timeseries | (uintptr_t)spectrum) & 7 || (uintptr_t)scratch & 255)
        return set_error(JERK_EINVAL,
                         "jerk_realfft: series and spectrum must be 8-byte aligned, scratch 256");
    if (scratch_bytes < (long long)rf_scratch(R1, R2))
        return set_error(JERK_EINVAL, "jerk_realfft: scratch smaller than jerk_realfft_scratch_bytes");
    cudaStream_t st = (cudaStream_t)stream;
    unsigned char *base = (unsigned char *)scratch;
    float2 *a = (float2 *)base;
    float2 *tw1 = (float2 *)(base + align256(sizeof(float2) * (size_t)R1 * R2));
    float2 *tw2 = (float2 *)((unsigned char *)tw1 + align256(sizeof(float2) * rf_twsize(R1)));
    float2 *out = (float2 *)spectrum;
    cudaError_t e = rf_dispatch<RfTw>(R1, tw1, st);
    if (e == cudaSuccess)
        e = rf_dispatch<RfTw>(R2, tw2, st);
    if (e == cudaSuccess)
        e = rf_dispatch<RfCol>(R1, (const float2 *)timeseries, R2, (const float2 *)tw1, a, st);
    if (e == cudaSuccess)
        e = rf_dispatch<RfRow>(R2, (const float2 *)a, R1, (const float2 *)tw2, out, st);
    if (e == cudaSuccess) {
        const long long M = (long long)R1 * R2;
        const long long threads = M / 2 + 1;
        const int grid = (int)std::min<long long>((threads + 255) / 256, 148LL * 16);
        rf_post_kernel<<<grid, 256, 0, st>>>(out, M);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess)
        return set_error(JERK_ECUDA, cudaGetErrorString(e));
    return JERK_OK;
}

extern "C" long long jerk_deredden_scratch_bytes(long long numamps)
{
    if (numamps < 8 || numamps > 0x7fffffffLL)
        return 0;
    return (long long)dr_scratch((int)numamps);
}

namespace {
int deredden_impl(void *spectrum, long long numamps, void *scratch, long long scratch_bytes,
                  void *stream, float bin0_imag)
{
    if (numamps < 8 || numamps > 0x7fffffffLL)
        return set_error(JERK_EINVAL, "jerk_deredden: numamps must be 8 .. 2^31-1");
    if (!spectrum || !scratch)
        return set_error(JERK_EINVAL, "jerk_deredden: null pointer");
    if ((uintptr_t)spectrum & 7 || (uintptr_t)scratch & 3)
        return set_error(JERK_EINVAL, "jerk_deredden: misaligned spectrum or scratch");
    if (scratch_bytes < (long long)dr_scratch((int)numamps))
        return set_error(JERK_EINVAL,
                         "jerk_deredden: scratch smaller than jerk_deredden_scratch_bytes");
    DrRuns runs;
    const int nb = dr_layout((int)numamps, &runs);
    if (nb < 1)
        return set_error(JERK_EUNSUPPORTED, "jerk_deredden: block layout too long");
    cudaStream_t st = (cudaStream_t)stream;
    float *level = (float *)scratch;
    float2 *x = (float2 *)spectrum;
    const int threads = 32 * kDrWarps;
    dr_level_kernel<<<(nb + kDrWarps - 1) / kDrWarps, threads, 0, st>>>(x, runs, nb, std::log(2.0),
                                                                       level);
    dr_scale_kernel<<<(nb + 1 + kDrWarps - 1) / kDrWarps, threads, 0, st>>>(
        x, runs, nb, (int)numamps, level, bin0_imag);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return set_error(JERK_ECUDA, cudaGetErrorString(e));
    return JERK_OK;
}
}  // namespace

// deredden sets bin 0 to (1, 0) (src/accel_utils.c:1569-1570).
extern "C" int jerk_deredden(void *spectrum, long long numamps, void *scratch,
                             long long scratch_bytes, void *stream)
{
    return deredden_impl(spectrum, numamps, scratch, scratch_bytes, stream, 0.0f);
}

extern "C" long long jerk_spectrum_scratch_bytes(long long n)
{
    const long long a = jerk_realfft_scratch_bytes(n), b = jerk_deredden_scratch_bytes(n / 2);
    return a && b ? std::max(a, b) : 0;
}

extern "C" int jerk_spectrum_from_timeseries(const float *timeseries, long long n, void *spectrum,
                                             void *scratch, long long scratch_bytes, void *stream)
{
    const int rc = jerk_realfft(timeseries, n, spectrum, scratch, scratch_bytes, stream);
    if (rc != JERK_OK)
        return rc;
    // create_accelobs then sets bin 0 of a .dat input to (1, 1) when the
    // powers are not photon-normalised (src/accel_utils.c:1829-1834)
    return deredden_impl(spectrum, n / 2, scratch, scratch_bytes, stream, 1.0f);
}

// The caller's loop around zapbirds (src/accelsearch_lib.c:393-418): birdies
// in list order, stopping at the first one at or above N/2, high edges
// clamped to N/2 - 1; birdies at or below 1.5 * 200 + 1 bins are left alone.
extern "C" int jerk_zap_birdies(void *spectrum, long long numbins, long long N,
                                const double *lobins, const double *hibins, int nbirds,
                                void *stream)
{
    if (!spectrum || numbins < 1 || N < 2 || nbirds < 0 || (nbirds && (!lobins || !hibins)))
        return set_error(JERK_EINVAL, "jerk_zap_birdies: bad argument");
    if ((uintptr_t)spectrum & 7)
        return set_error(JERK_EINVAL, "jerk_zap_birdies: misaligned spectrum");
    cudaStream_t st = (cudaStream_t)stream;
    const double top = (double)(N / 2);
    const double neg_log_half = -std::log(0.5);
    for (int i = 0; i < nbirds; i++) {
        if (lobins[i] >= top)
            break;
        const double lo = lobins[i], hi = hibins[i] >= top ? top - 1 : hibins[i];
        if (!(lo - 1.5 * kZapBins > 1))
            continue;
        zap_kernel<<<1, kZapThreads, 0, st>>>((float2 *)spectrum, numbins, lo, hi, neg_log_half);
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return set_error(JERK_ECUDA, cudaGetErrorString(e));
    return JERK_OK;
}
