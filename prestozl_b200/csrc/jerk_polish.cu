// Candidate polishing on the GPU: the volume search of the reference's
// harmonic polishing (max_rzw_arr_harmonics, src/maximize_rzw.c:84-190, the
// default optimisation of optimize_accelcand, src/accel_utils.c:573-657).
//
// For a candidate (r, z, w) with numharm harmonics, the reference builds, per
// harmonic n = numharm .. 1 (highest first), an oversampled
// f / f-dot / f-dotdot volume around (n r, n z, n w) with corr_rzw_vol
// (src/rzwinterp.c:3-148): 17 x 17 (w, z) response kernels at 8 points per
// bin (gen_w_response, src/responses.c:333-418, or gen_z/gen_r_response
// where w ~ 0), each placed and FFT'd, correlated with the raw spectrum
// around the harmonic (corr_complex, src/corr_routines.c: spread by 8, FFT,
// times conj(kernel) / fftlen, inverse FFT, kern_half_width * 8 points
// chopped).  The powers at 24 r positions on the fundamental's grid, each
// over the harmonic's local power, are summed across harmonics; the first
// strict maximum in (w, z, r) order gives the polished (r, z, w).
//
// Here one call does the whole volume search of one candidate on the GPU:
//   pzr_response_kernel      w ~ 0 rows: z responses (Fresnel integrals) or
//                            the interbin sinc, in double, rounded to float
//   pw_response_kernel<M>    w rows: the reference's float cosine series of
//                            npts samples, zero-padded to 8 npts, real FFT
//                            (an M = 4 npts point complex FFT in shared memory
//                            and the real split of the numkern bins needed)
//   pk_fft_kernel<N>         forward FFT of every kernel row, in place
//   pd_data_kernel<N>        each harmonic's data window spread by 8, FFT'd
//   pc_corr_kernel<N>        per kernel row: times conj(kernel) / fftlen,
//                            inverse FFT, power at the 24 r positions over
//                            the local power
//   ps_argmax_kernel         sum over harmonics in the reference's order,
//                            first strict maximum
// The local powers (get_localpower3d, src/characteristics.c:75-135) come in
// from the caller, which computes them as the reference does.  FP32 FFTs
// like the reference's FFTW, so the volume powers agree to FP32 rounding and
// the chosen grid point is the reference's unless two grid powers tie to
// that rounding.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "jerk.h"
#include "jerk_fft.cuh"
#include "jerk_kernels.cuh"
#include "jerk_resp.cuh"

namespace jerk {
namespace {

constexpr int kNb = 8;                            // numbetween: interpfac 4 x ACCEL_RDR 2
constexpr int kInterp = 4;                        // interpfac
constexpr int kNumWid = 2;                        // numwid
constexpr int kGrid = 2 * kNumWid * kInterp + 1;  // 17 z and 17 w values
constexpr int kCells = kGrid * kGrid;             // kernels per harmonic
constexpr int kNumR = 3 * kNb;                    // 24 r values
constexpr int kWin = 40;                          // r positions kept per row (>= span of rind)
constexpr double kDZ = 2.0, kDW = 20.0;           // ACCEL_DZ, ACCEL_DW
constexpr int kMaxHarm = 32;
// Where rind < 0 the reference reads vol[w][z][rind] past the start of the
// (w, z) row: the contiguous volume gives it the previous row's last good
// values (for the first row, allocator bytes before the array: taken as 0).
// Realistic candidates reach rind = -3; rows keep their last kTail powers.
constexpr int kTail = 4;
constexpr int kMinFft = 128, kMaxFft = 8192;      // kernel rows, data windows
constexpr int kMinM = 128, kMaxM = 8192;          // w-response FFTs

struct PolishHarm {
    long long row0;   // index of this harmonic's first row
    long long data;   // float2 offset of its FFT'd data window
    long long win;    // float2 offset of its staged raw window
    int fftlen, khw, numkern;
    int numgood;      // good volume values per (w, z) row
    int rmin;         // smallest rind (>= -kTail)
    int rind[kNumR];  // volume index of each r of the fundamental's grid
    float locpow;
};

struct PolishRow {
    long long off;  // float2 offset of the kernel row
    double z, w;
    int fftlen, numkern, npts, harm;
};

// ---------------------------------------------------------------------------
// responses

constexpr int kRespThreads = 256;

// w ~ 0: gen_z_response (src/responses.c:228-313) or, for z ~ 0 too,
// gen_r_response (src/responses.c:158-226), roffset 0, numbetween kNb.
__global__ void __launch_bounds__(kRespThreads)
    pzr_response_kernel(const PolishRow *__restrict__ rows, const int *__restrict__ list,
                        float2 *__restrict__ bank)
{
    const PolishRow R = rows[list[blockIdx.x]];
    const int tid = threadIdx.x;
    float2 *row = bank + R.off;
    const int numkern = R.numkern;
    for (int m = numkern / 2 + tid; m < R.fftlen - numkern / 2; m += kRespThreads)
        row[m] = make_float2(0.f, 0.f);
    const double z = R.z;
    if (fabs(z) >= 1e-4) {
        const double absz = fabs(z);
        const double startr0 = -(0.5 * z);
        double ipart;
        const double startroffset =
            startr0 < 0.0 ? 1.0 + modf(startr0, &ipart) : modf(startr0, &ipart);
        const int signz = z < 0.0 ? -1 : 1;
        const double zd = signz * 1.4142135623730950488016887242096980785696718753769 / sqrt(absz);
        const double cons = zd / 2.0;
        const double pibyz = M_PI / z;
        const double startr = startr0 + numkern / (double)(2 * kNb);
        const double delta = -1.0 / kNb;
        for (int ii = tid; ii < numkern; ii += kRespThreads) {
            const double r = __dadd_rn(startr, __dmul_rn((double)ii, delta));
            const double yy = __dmul_rn(r, zd);
            const double zz = __dadd_rn(yy, __dmul_rn(z, zd));
            const double xx = __dmul_rn(__dmul_rn(pibyz, r), r);
            double sn, cs, fsy, fcy, fsz, fcz;
            sincos(xx, &sn, &cs);
            fresnel(yy, &fsy, &fcy);
            fresnel(zz, &fsz, &fcz);
            const double tmprl = signz * (fcz - fcy);
            const double tmpim = fsy - fsz;
            float re = (float)__dmul_rn(__dsub_rn(__dmul_rn(tmprl, cs), __dmul_rn(tmpim, sn)), cons);
            float im = (float)-__dmul_rn(__dadd_rn(__dmul_rn(tmprl, sn), __dmul_rn(tmpim, cs)), cons);
            if (ii == numkern / 2 && startroffset < 1e-3 && absz < 1e-3) {
                // the reference's series at the centre point (src/responses.c:297-310)
                const double z2 = z * z, x2 = startroffset * startroffset;
                double cr = 1.0 - 0.16449340668482264365 * z2;
                double ci = -0.5235987755982988731 * z;
                cr += startroffset * 1.6449340668482264365 * z;
                ci += startroffset * (M_PI - 0.5167712780049970029 * z2);
                cr += x2 * (-6.579736267392905746 + 0.9277056288952613070 * z2);
                ci += x2 * (3.1006276680299820175 * z);
                re = (float)cr;
                im = (float)ci;
            }
            row[placed(ii, numkern, R.fftlen)] = make_float2(re, im);
        }
    } else {
        // value ii = exp(i r) sin(r) / r at r = pi (numkern / (2 nb) - ii / nb)
        for (int ii = tid; ii < numkern; ii += kRespThreads) {
            const double q = numkern / (double)(2 * kNb) - ii / (double)kNb;  // r / pi
            float re = 1.0f, im = 0.0f;
            if (q != 0.0) {
                double sn, cs;
                sincospi(q, &sn, &cs);
                const double sinc = sn / (M_PI * q);
                re = (float)(cs * sinc);
                im = (float)(sn * sinc);
            }
            row[placed(ii, numkern, R.fftlen)] = make_float2(re, im);
        }
    }
}

// w != 0: gen_w_response (src/responses.c:333-418), roffset 0.  The series
// x[n] = (float)(amp cos(phase(n))), n < npts, zero-padded to L = 8 npts,
// is read as M = L / 2 complex values; after the M-point FFT the response
// bins kc = M/2 - numkern/2 + k (k < numkern) come from the real split of
// Z[kc] and Z[M - kc], both inside the window Z[M/2 - numkern/2 ..
// M/2 + numkern/2], which the last FFT stage drops into shared memory.
template <int M>
__global__ void __launch_bounds__(FftPlan<M>::T)
    pw_response_kernel(const PolishRow *__restrict__ rows, const int *__restrict__ list,
                       const float2 *__restrict__ tw, float2 *__restrict__ bank)
{
    constexpr int T = FftPlan<M>::T;
    extern __shared__ float2 pw_smem[];
    float2 *buf = pw_smem;
    float2 *win = pw_smem + fft_buf_len<M>();
    const PolishRow R = rows[list[blockIdx.x]];
    const int tid = threadIdx.x;
    float2 *row = bank + R.off;
    const int numkern = R.numkern;
    const int npts = R.npts;
    const double z = R.z, w = R.w;
    const double dt = 1.0 / (double)npts;
    const double amp = 2.0 * dt;
    const int fbar = npts / 4;
    const double f = __dadd_rn(__dsub_rn((double)fbar, 0.5 * z), w / 12.0);
    const double fd = (z - 0.5 * w) / 2.0;
    const double fdd = w / 6.0;
    auto xval = [&](int n) -> float {
        if (n >= npts)
            return 0.0f;
        const double t = __dmul_rn((double)n, dt);
        const double in1 = __dadd_rn(__dmul_rn(t, fdd), fd);
        const double in2 = __dadd_rn(__dmul_rn(t, in1), f);
        const double ph = __dmul_rn(6.2831853071795864769252867665590057683943387987502,
                                    __dmul_rn(t, in2));
        return (float)__dmul_rn(amp, cos(ph));
    };
    auto in = [&](int r) -> float2 {
        const int m = tid + r * T;
        return make_float2(xval(2 * m), xval(2 * m + 1));
    };
    const int lo = M / 2 - numkern / 2;
    auto out = [&](int k, float2 y) {
        if (k >= lo && k <= lo + numkern)
            win[k - lo] = y;
    };
    fft_block<M, -1>(buf, tw, tid, in, out);
    for (int m = numkern / 2 + tid; m < R.fftlen - numkern / 2; m += T)
        row[m] = make_float2(0.f, 0.f);
    __syncthreads();
    for (int k = tid; k < numkern; k += T) {
        const int kc = lo + k;
        const float2 a = win[k], b = win[numkern - k];  // Z[kc], Z[M - kc]
        const double hx = 0.5 * ((double)a.x + (double)b.x);
        const double hy = 0.5 * ((double)a.y - (double)b.y);
        const double dx = (double)a.x - (double)b.x;
        const double dy = (double)a.y + (double)b.y;
        double s, c;
        sincospi(-(double)kc / (double)M, &s, &c);
        const double gx = c * dx - s * dy, gy = c * dy + s * dx;
        row[placed(k, numkern, R.fftlen)] =
            make_float2((float)(hx + 0.5 * gy), (float)(hy - 0.5 * gx));
    }
}

// ---------------------------------------------------------------------------
// kernel-row FFTs, data windows, correlations

template <int N>
__global__ void __launch_bounds__(FftPlan<N>::T)
    pk_fft_kernel(const PolishRow *__restrict__ rows, int first, const float2 *__restrict__ tw,
                  float2 *__restrict__ bank)
{
    constexpr int T = FftPlan<N>::T;
    extern __shared__ float2 pk_buf[];
    float2 *row = bank + rows[first + blockIdx.x].off;
    const int tid = threadIdx.x;
    auto in = [&](int r) -> float2 { return row[tid + r * T]; };
    auto out = [&](int m, float2 y) { row[m] = y; };
    fft_block<N, -1>(pk_buf, tw, tid, in, out);
}

// spread_no_pad (src/corr_prep.c:37-74) by 8, then the forward FFT
template <int N>
__global__ void __launch_bounds__(FftPlan<N>::T)
    pd_data_kernel(const PolishHarm *__restrict__ harms, int first, const float2 *__restrict__ tw,
                   const float2 *__restrict__ windows, float2 *__restrict__ dfft)
{
    constexpr int T = FftPlan<N>::T;
    extern __shared__ float2 pd_buf[];
    const PolishHarm H = harms[first + blockIdx.x];
    const float2 *src = windows + H.win;
    float2 *dst = dfft + H.data;
    const int tid = threadIdx.x;
    auto in = [&](int r) -> float2 {
        const int m = tid + r * T;
        return (m % kNb) == 0 ? src[m / kNb] : make_float2(0.f, 0.f);
    };
    auto out = [&](int m, float2 y) { dst[m] = y; };
    fft_block<N, -1>(pd_buf, tw, tid, in, out);
}

// complex_corr_conv (src/correlations.c:3-55, CORR) and the chop of
// corr_complex: amplitude i of the volume is y[khw * 8 + i]
template <int N>
__global__ void __launch_bounds__(FftPlan<N>::T)
    pc_corr_kernel(const PolishRow *__restrict__ rows, int first,
                   const PolishHarm *__restrict__ harms, const float2 *__restrict__ tw,
                   const float2 *__restrict__ bank, const float2 *__restrict__ dfft,
                   float *__restrict__ terms, float *__restrict__ tails)
{
    constexpr int T = FftPlan<N>::T;
    extern __shared__ float2 pc_buf[];
    __shared__ float pw[kWin];
    const int rowi = first + blockIdx.x;
    const PolishRow R = rows[rowi];
    const PolishHarm &H = harms[R.harm];
    const float2 *krow = bank + R.off;
    const float2 *d = dfft + H.data;
    const int tid = threadIdx.x;
    const float normal = 1.0f / (float)N;
    auto in = [&](int r) -> float2 {
        const int m = tid + r * T;
        const float2 a = d[m], k = krow[m];
        return make_float2(__fmul_rn(__fadd_rn(__fmul_rn(a.x, k.x), __fmul_rn(a.y, k.y)), normal),
                           __fmul_rn(__fsub_rn(__fmul_rn(a.y, k.x), __fmul_rn(k.y, a.x)), normal));
    };
    const int base = H.khw * kNb + H.rmin;
    const int tail0 = H.khw * kNb + H.numgood - kTail;
    auto out = [&](int m, float2 y) {
        const float p = __fadd_rn(__fmul_rn(y.x, y.x), __fmul_rn(y.y, y.y));
        const int i = m - base;
        if (i >= 0 && i < kWin)
            pw[i] = p;
        const int t = m - tail0;
        if (t >= 0 && t < kTail)
            tails[(long long)rowi * kTail + t] = p;
    };
    fft_block<N, +1>(pc_buf, tw, tid, in, out);
    __syncthreads();
    if (tid < kNumR && H.rind[tid] >= 0)
        terms[(long long)rowi * kNumR + tid] = __fdiv_rn(pw[H.rind[tid] - H.rmin], H.locpow);
}

// powsum[w][z][r] = sum over harmonics (highest first) of the terms; the first
// strict maximum above 0 in (w, z, r) order.  One CTA.
constexpr int kArgThreads = 1024;
__global__ void __launch_bounds__(kArgThreads)
    ps_argmax_kernel(const float *__restrict__ terms, const float *__restrict__ tails,
                     const PolishHarm *__restrict__ harms, int numharm, int *__restrict__ best,
                     float *__restrict__ bestpow)
{
    __shared__ float sv[kArgThreads / 32];
    __shared__ int si[kArgThreads / 32];
    const int tid = threadIdx.x;
    float bv = 0.0f;
    int bi = 0x7fffffff;
    for (int c = tid; c < kCells * kNumR; c += kArgThreads) {
        const int cell = c / kNumR, kk = c % kNumR;
        float s = 0.0f;
        for (int h = 0; h < numharm; h++) {
            const int ri = harms[h].rind[kk];
            const long long row = (long long)h * kCells + cell;
            float t;
            if (ri >= 0)
                t = terms[row * kNumR + kk];
            else if (cell > 0)
                t = __fdiv_rn(tails[(row - 1) * kTail + kTail + ri], harms[h].locpow);
            else
                t = 0.0f;
            s = __fadd_rn(s, t);
        }
        if (s > bv) {  // cells visited in increasing order per thread
            bv = s;
            bi = c;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const float ov = __shfl_down_sync(0xffffffffu, bv, o);
        const int oi = __shfl_down_sync(0xffffffffu, bi, o);
        if (ov > bv || (ov == bv && oi < bi)) {
            bv = ov;
            bi = oi;
        }
    }
    if ((tid & 31) == 0) {
        sv[tid >> 5] = bv;
        si[tid >> 5] = bi;
    }
    __syncthreads();
    if (tid < 32) {
        bv = sv[tid];
        bi = si[tid];
        for (int o = 16; o > 0; o >>= 1) {
            const float ov = __shfl_down_sync(0xffffffffu, bv, o);
            const int oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (ov > bv || (ov == bv && oi < bi)) {
                bv = ov;
                bi = oi;
            }
        }
        if (tid == 0) {
            *best = bi == 0x7fffffff ? 0 : bi;
            *bestpow = bv;
        }
    }
}

// per-stage twiddles of every power-of-two plan 128..8192, in double
template <int N, int S>
__device__ __forceinline__ void p_stage_twiddle(int i, float2 *tw)
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
            p_stage_twiddle<N, S + 1>(i, tw);
        }
    }
}
template <int N>
__global__ void p_twiddle_kernel(float2 *tw)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < FftPlan<N>::twsize())
        p_stage_twiddle<N, 1>(i, tw);
}

constexpr int kSizes[] = {128, 256, 512, 1024, 2048, 4096, 8192};
constexpr int kNumSizes = 7;
int size_index(int n)
{
    for (int i = 0; i < kNumSizes; i++)
        if (kSizes[i] == n)
            return i;
    return -1;
}
template <int N>
constexpr int tw_size()
{
    return FftPlan<N>::twsize();
}
int tw_size_rt(int n)
{
    switch (n) {
    case 128: return tw_size<128>();
    case 256: return tw_size<256>();
    case 512: return tw_size<512>();
    case 1024: return tw_size<1024>();
    case 2048: return tw_size<2048>();
    case 4096: return tw_size<4096>();
    case 8192: return tw_size<8192>();
    default: return 0;
    }
}

template <template <int> class F, class... A>
cudaError_t p_dispatch(int n, A... args)
{
    switch (n) {
    case 128: return F<128>::run(args...);
    case 256: return F<256>::run(args...);
    case 512: return F<512>::run(args...);
    case 1024: return F<1024>::run(args...);
    case 2048: return F<2048>::run(args...);
    case 4096: return F<4096>::run(args...);
    case 8192: return F<8192>::run(args...);
    default: return cudaErrorInvalidValue;
    }
}

template <int N> struct PTw {
    static cudaError_t run(float2 *tw, cudaStream_t st)
    {
        p_twiddle_kernel<N><<<(tw_size<N>() + 255) / 256, 256, 0, st>>>(tw);
        return cudaGetLastError();
    }
};
template <int M> struct PW {
    static cudaError_t run(const PolishRow *rows, const int *list, int count, const float2 *tw,
                           float2 *bank, int maxkern, cudaStream_t st)
    {
        const int smem = (int)(sizeof(float2) * (fft_buf_len<M>() + maxkern + 1));
        cudaError_t e = cudaFuncSetAttribute(pw_response_kernel<M>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess)
            return e;
        pw_response_kernel<M><<<count, FftPlan<M>::T, smem, st>>>(rows, list, tw, bank);
        return cudaGetLastError();
    }
};
template <int N> struct PK {
    static cudaError_t run(const PolishRow *rows, int first, int count, const float2 *tw,
                           float2 *bank, cudaStream_t st)
    {
        const int smem = (int)(sizeof(float2) * fft_buf_len<N>());
        cudaError_t e = cudaFuncSetAttribute(pk_fft_kernel<N>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess)
            return e;
        pk_fft_kernel<N><<<count, FftPlan<N>::T, smem, st>>>(rows, first, tw, bank);
        return cudaGetLastError();
    }
};
template <int N> struct PD {
    static cudaError_t run(const PolishHarm *harms, int first, int count, const float2 *tw,
                           const float2 *windows, float2 *dfft, cudaStream_t st)
    {
        const int smem = (int)(sizeof(float2) * fft_buf_len<N>());
        cudaError_t e = cudaFuncSetAttribute(pd_data_kernel<N>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess)
            return e;
        pd_data_kernel<N><<<count, FftPlan<N>::T, smem, st>>>(harms, first, tw, windows, dfft);
        return cudaGetLastError();
    }
};
template <int N> struct PC {
    static cudaError_t run(const PolishRow *rows, int first, int count, const PolishHarm *harms,
                           const float2 *tw, const float2 *bank, const float2 *dfft,
                           float *terms, float *tails, cudaStream_t st)
    {
        const int smem = (int)(sizeof(float2) * fft_buf_len<N>());
        cudaError_t e = cudaFuncSetAttribute(pc_corr_kernel<N>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess)
            return e;
        pc_corr_kernel<N><<<count, FftPlan<N>::T, smem, st>>>(rows, first, harms, tw, bank, dfft,
                                                              terms, tails);
        return cudaGetLastError();
    }
};

long long next2(long long x)
{
    long long n = 1;
    while (n < x)
        n <<= 1;
    return n;
}

// One run of spectrum values read from a spectrum held on the device:
// count values from index src (zero outside [0, numdata)) to dst[off] with
// dst = the windows, or the answers where to_ans is set.
struct WinSeg {
    long long src, off;
    int count, to_ans;
};

constexpr int kGatherThreads = 128;

__global__ void __launch_bounds__(kGatherThreads)
gather_windows_kernel(const float2 *__restrict__ spec, long long numdata,
                      const WinSeg *__restrict__ segs, float2 *__restrict__ win,
                      float2 *__restrict__ ans)
{
    const WinSeg s = segs[blockIdx.x];
    float2 *dst = (s.to_ans ? ans : win) + s.off;
    for (int i = threadIdx.x; i < s.count; i += kGatherThreads) {
        const long long b = s.src + i;
        dst[i] = (b >= 0 && b < numdata) ? spec[b] : make_float2(0.f, 0.f);
    }
}

// Where the spectrum lives: device (or managed) memory is read on the GPU by
// gather_windows_kernel, anything else on the host.
bool spectrum_on_device(const void *spectrum)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, spectrum) != cudaSuccess) {
        cudaGetLastError();  // a plain host pointer on an old runtime
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace
}  // namespace jerk

using namespace jerk;

// Device buffers grow to the largest candidate seen and are kept.
struct jerk_polisher {
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    float2 *tw = nullptr;
    int twoff[kNumSizes] = {};
    float2 *bank = nullptr;
    long long bank_cap = 0;
    float2 *dfft = nullptr, *windows = nullptr;
    long long dfft_cap = 0, win_cap = 0;
    float *terms = nullptr, *tails = nullptr;
    long long terms_cap = 0, tails_cap = 0;
    PolishRow *d_rows = nullptr;
    int *d_lists = nullptr;
    long long rows_cap = 0, lists_cap = 0;
    WinSeg *d_segs = nullptr;  // window runs of a spectrum held on the device
    long long segs_cap = 0;
    PolishHarm *d_harms = nullptr;
    int *d_best = nullptr;
    float *d_bestpow = nullptr;
    // pinned staging: rows, lists, harms, windows
    unsigned char *h_stage = nullptr;
    long long stage_cap = 0;
    long long candidates = 0;
};

namespace {

int p_fail(int code, const char *msg) { return set_error(code, msg); }

int p_cuda(cudaError_t e, const char *what)
{
    static thread_local char buf[256];
    snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    return set_error(JERK_ECUDA, buf);
}

template <class T>
cudaError_t grow(T **p, long long *cap, long long need)
{
    if (need <= *cap)
        return cudaSuccess;
    const long long n = std::max(need, *cap * 3 / 2);
    if (*p)
        cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    cudaError_t e = cudaMalloc(p, sizeof(T) * (size_t)n);
    if (e == cudaSuccess)
        *cap = n;
    return e;
}

}  // namespace

extern "C" int jerk_polisher_create(jerk_polisher **out, void *stream)
{
    if (!out)
        return p_fail(JERK_EINVAL, "jerk_polisher_create: null pointer");
    jerk_polisher *p = new jerk_polisher();
    cudaError_t e = cudaSuccess;
    if (stream) {
        p->stream = (cudaStream_t)stream;
    } else {
        e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking);
        p->own_stream = true;
    }
    int total = 0;
    for (int i = 0; i < kNumSizes; i++) {
        p->twoff[i] = total;
        total += tw_size_rt(kSizes[i]);
    }
    if (e == cudaSuccess)
        e = cudaMalloc(&p->tw, sizeof(float2) * total);
    for (int i = 0; i < kNumSizes && e == cudaSuccess; i++)
        e = p_dispatch<PTw>(kSizes[i], p->tw + p->twoff[i], p->stream);
    if (e == cudaSuccess)
        e = cudaMalloc(&p->d_harms, sizeof(PolishHarm) * kMaxHarm);
    if (e == cudaSuccess)
        e = cudaMalloc(&p->d_best, sizeof(int));
    if (e == cudaSuccess)
        e = cudaMalloc(&p->d_bestpow, sizeof(float));
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(p->stream);
    if (e != cudaSuccess) {
        jerk_polisher_destroy(p);
        return p_cuda(e, "jerk_polisher_create");
    }
    *out = p;
    return JERK_OK;
}

extern "C" void jerk_polisher_destroy(jerk_polisher *p)
{
    if (!p)
        return;
    if (p->stream)
        cudaStreamSynchronize(p->stream);
    cudaFree(p->tw);
    cudaFree(p->bank);
    cudaFree(p->dfft);
    cudaFree(p->windows);
    cudaFree(p->terms);
    cudaFree(p->tails);
    cudaFree(p->d_rows);
    cudaFree(p->d_lists);
    cudaFree(p->d_segs);
    cudaFree(p->d_harms);
    cudaFree(p->d_best);
    cudaFree(p->d_bestpow);
    if (p->h_stage)
        cudaFreeHost(p->h_stage);
    if (p->own_stream && p->stream)
        cudaStreamDestroy(p->stream);
    delete p;
}

// The host side of one candidate: per-harmonic geometry as
// max_rzw_arr_harmonics and corr_rzw_vol compute it (src/maximize_rzw.c:104-140,
// src/rzwinterp.c:42-61), one row per (harmonic, w, z) kernel, and the row
// lists by response kind and FFT size.
struct PolishPlan {
    std::vector<PolishHarm> harms;
    std::vector<PolishRow> rows;
    std::vector<int> lists;  // w ~ 0 rows, then w rows by M
    int nzr = 0;
    int mfirst[kNumSizes] = {}, mcount[kNumSizes] = {}, maxkern[kNumSizes] = {};
    long long hhlobin = 0, bank_len = 0, dfft_len = 0, win_len = 0;
};

int polish_plan(int numharm, double rin, double zin, double win, long long numdata,
                const float *locpow, PolishPlan &out)
{
    const double dr = 1.0 / (double)kNb;

    // ---- host: per-harmonic geometry (src/maximize_rzw.c:104-140, src/rzwinterp.c:42-61)
    out = PolishPlan();
    std::vector<PolishHarm> &H = out.harms;
    std::vector<PolishRow> &rows = out.rows;
    H.resize(numharm);
    rows.reserve((size_t)numharm * kCells);
    long long hhlobin = 0, bank_len = 0, dfft_len = 0, win_len = 0;
    int *maxkern = out.maxkern;
    for (int hind = 0; hind < numharm; hind++) {
        const int n = numharm - hind;
        const double rh = rin * n, zh = zin * n, wh = win * n;
        const int khw_c = w_resp_halfwidth_lowacc(fabs(zh) + 2, fabs(wh) + 20);
        const double hfrac = n / (double)numharm;
        double rh_int;
        modf(rh, &rh_int);
        const long long lobin = (long long)rh_int - 1;
        if (hind == 0)
            hhlobin = lobin;
        const long long fftlen = next2(kNb * (2 * khw_c + 10));
        if (fftlen < kMinFft || fftlen > kMaxFft)
            return p_fail(JERK_EUNSUPPORTED, "jerk_polish_rzw: correlation length beyond 8192");
        const double zlo = zh - kNumWid * hfrac * kDZ, zhi = zh + kNumWid * hfrac * kDZ;
        const double wlo = wh - kNumWid * hfrac * kDW, whi = wh + kNumWid * hfrac * kDW;
        const double dz = (zhi - zlo) / (kGrid - 1), dw = (whi - wlo) / (kGrid - 1);
        const double maxz = fabs(zlo) < fabs(zhi) ? zhi : zlo;
        const double maxw = fabs(wlo) < fabs(whi) ? whi : wlo;
        const int khw = w_resp_halfwidth_lowacc(maxz, maxw);
        const int numkern = 2 * kNb * khw;
        int numgood = (int)fftlen - 2 * khw * kNb;
        while (numgood > 0 && numgood % kNb)
            numgood--;
        if (lobin < 0 || lobin >= numdata)
            return p_fail(JERK_EINVAL, "jerk_polish_rzw: harmonic outside the spectrum");
        PolishHarm &h = H[hind];
        h.fftlen = (int)fftlen;
        h.khw = khw;
        h.numkern = numkern;
        h.locpow = locpow[hind];
        h.numgood = numgood;
        if (numgood < kTail)
            return p_fail(JERK_EUNSUPPORTED, "jerk_polish_rzw: volume narrower than its r grid");
        int rmin = 1 << 30, rmax = -1;
        for (int kk = 0; kk < kNumR; kk++) {
            const long long ri =
                (long long)round(((hhlobin + kk * dr) * hfrac - lobin) * kNb);
            if (ri < -kTail || ri >= numgood)
                return p_fail(JERK_EUNSUPPORTED, "jerk_polish_rzw: r grid outside the volume");
            h.rind[kk] = (int)ri;
            rmin = std::min(rmin, (int)ri);
            rmax = std::max(rmax, (int)ri);
        }
        if (rmax - rmin >= kWin)
            return p_fail(JERK_EUNSUPPORTED, "jerk_polish_rzw: r grid wider than expected");
        h.rmin = rmin;
        h.row0 = (long long)rows.size();
        h.data = dfft_len;
        h.win = win_len;
        dfft_len += fftlen;
        win_len += fftlen / kNb;
        for (int ii = 0; ii < kGrid; ii++)
            for (int jj = 0; jj < kGrid; jj++) {
                PolishRow R{};
                R.off = bank_len;
                bank_len += fftlen;
                R.z = zlo + jj * dz;
                R.w = wlo + ii * dw;
                R.fftlen = (int)fftlen;
                R.numkern = numkern;
                R.harm = hind;
                R.npts = 0;
                if (fabs(R.w) >= 1e-4) {
                    R.npts = (int)next2(6 * w_resp_halfwidth_lowacc(R.z, R.w) + 200 + numkern / kNb);
                    const long long M = (long long)R.npts * kNb / 2;
                    if (M < kMinM || M > kMaxM || numkern / 2 >= M / 2)
                        return p_fail(JERK_EUNSUPPORTED,
                                      "jerk_polish_rzw: w response FFT beyond 8192 points");
                    const int mi = size_index((int)M);
                    maxkern[mi] = std::max(maxkern[mi], numkern);
                }
                rows.push_back(R);
            }
    }
    const long long nrows = (long long)rows.size();

    // row lists: w ~ 0 rows, then w rows grouped by M
    std::vector<int> &lists = out.lists;
    lists.reserve(nrows);
    for (long long i = 0; i < nrows; i++)
        if (rows[i].npts == 0)
            lists.push_back((int)i);
    const int nzr = (int)lists.size();
    int *mfirst = out.mfirst, *mcount = out.mcount;
    for (int s = 0; s < kNumSizes; s++) {
        mfirst[s] = (int)lists.size();
        for (long long i = 0; i < nrows; i++)
            if (rows[i].npts && (long long)rows[i].npts * kNb / 2 == kSizes[s])
                lists.push_back((int)i);
        mcount[s] = (int)lists.size() - mfirst[s];
    }
    out.nzr = nzr;
    out.hhlobin = hhlobin;
    out.bank_len = bank_len;
    out.dfft_len = dfft_len;
    out.win_len = win_len;
    return JERK_OK;
}

extern "C" int jerk_polish_rzw(jerk_polisher *p, const void *spectrum, long long numdata,
                               int numharm, double rin, double zin, double win,
                               const float *locpow, double *rout, double *zout, double *wout,
                               float *maxpow)
{
    if (!p || !spectrum || !locpow || !rout || !zout || !wout)
        return p_fail(JERK_EINVAL, "jerk_polish_rzw: null pointer");
    if (numharm < 1 || numharm > kMaxHarm || numdata < 1)
        return p_fail(JERK_EINVAL, "jerk_polish_rzw: numharm must be 1..32, numdata > 0");
    const float2 *data = (const float2 *)spectrum;
    const double dr = 1.0 / (double)kNb;
    PolishPlan P;
    const int rc = polish_plan(numharm, rin, zin, win, numdata, locpow, P);
    if (rc != JERK_OK)
        return rc;
    std::vector<PolishHarm> &H = P.harms;
    std::vector<PolishRow> &rows = P.rows;
    std::vector<int> &lists = P.lists;
    const long long nrows = (long long)rows.size();
    const long long hhlobin = P.hhlobin, bank_len = P.bank_len, dfft_len = P.dfft_len,
                    win_len = P.win_len;
    const int nzr = P.nzr;
    const int *mfirst = P.mfirst, *mcount = P.mcount, *maxkern = P.maxkern;

    // ---- staging: rows | lists | harms | data windows (zero outside the
    // spectrum), or for a spectrum on the device the windows' runs in it
    const bool dev = spectrum_on_device(spectrum);
    const size_t b_rows = sizeof(PolishRow) * nrows, b_lists = sizeof(int) * lists.size();
    const size_t b_harms = sizeof(PolishHarm) * numharm;
    const size_t b_win = dev ? sizeof(WinSeg) * numharm : sizeof(float2) * win_len;
    const size_t o_win = (b_rows + b_lists + b_harms + 15) & ~(size_t)15;
    const long long stage = (long long)(o_win + b_win);
    cudaError_t e = cudaSuccess;
    if (stage > p->stage_cap) {
        if (p->h_stage)
            cudaFreeHost(p->h_stage);
        p->h_stage = nullptr;
        p->stage_cap = 0;
        e = cudaMallocHost(&p->h_stage, stage * 2);
        if (e != cudaSuccess)
            return p_cuda(e, "jerk_polish_rzw: pinned staging");
        p->stage_cap = stage * 2;
    }
    e = cudaStreamSynchronize(p->stream);  // the staging buffer is free again
    if (e != cudaSuccess)
        return p_cuda(e, "jerk_polish_rzw: stream");
    unsigned char *hs = p->h_stage;
    memcpy(hs, rows.data(), b_rows);
    memcpy(hs + b_rows, lists.data(), b_lists);
    memcpy(hs + b_rows + b_lists, H.data(), b_harms);
    float2 *hw = (float2 *)(hs + o_win);
    WinSeg *hseg = (WinSeg *)hw;
    for (int hind = 0; hind < numharm; hind++) {
        const PolishHarm &h = H[hind];
        const int n = numharm - hind;
        double rh_int;
        modf(rin * n, &rh_int);
        const long long begin = (long long)rh_int - 1 - h.khw;
        const int nb = h.fftlen / kNb;
        if (dev) {
            hseg[hind] = WinSeg{begin, h.win, nb, 0};
            continue;
        }
        for (int i = 0; i < nb; i++) {
            const long long b = begin + i;
            hw[h.win + i] = (b >= 0 && b < numdata) ? data[b] : make_float2(0.f, 0.f);
        }
    }
    if ((e = grow(&p->bank, &p->bank_cap, bank_len)) != cudaSuccess ||
        (e = grow(&p->dfft, &p->dfft_cap, dfft_len)) != cudaSuccess ||
        (e = grow(&p->windows, &p->win_cap, win_len)) != cudaSuccess ||
        (e = grow(&p->terms, &p->terms_cap, nrows * kNumR)) != cudaSuccess ||
        (e = grow(&p->tails, &p->tails_cap, nrows * kTail)) != cudaSuccess ||
        (e = grow(&p->d_rows, &p->rows_cap, nrows)) != cudaSuccess ||
        (e = grow(&p->d_lists, &p->lists_cap, (long long)lists.size())) != cudaSuccess ||
        (dev && (e = grow(&p->d_segs, &p->segs_cap, (long long)numharm)) != cudaSuccess))
        return p_cuda(e, "jerk_polish_rzw: device buffers");
    cudaStream_t st = p->stream;
    e = cudaMemcpyAsync(p->d_rows, hs, b_rows, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(p->d_lists, hs + b_rows, b_lists, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(p->d_harms, hs + b_rows + b_lists, b_harms, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dev ? (void *)p->d_segs : (void *)p->windows, hw, b_win,
                            cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && dev) {
        gather_windows_kernel<<<numharm, kGatherThreads, 0, st>>>(data, numdata, p->d_segs,
                                                                  p->windows, nullptr);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess)
        return p_cuda(e, "jerk_polish_rzw: upload");

    // ---- device: responses, kernel FFTs, data FFTs, correlations, sum and argmax
    if (nzr > 0) {
        pzr_response_kernel<<<nzr, kRespThreads, 0, st>>>(p->d_rows, p->d_lists, p->bank);
        e = cudaGetLastError();
    }
    for (int s = 0; s < kNumSizes && e == cudaSuccess; s++)
        if (mcount[s])
            e = p_dispatch<PW>(kSizes[s], (const PolishRow *)p->d_rows,
                               (const int *)p->d_lists + mfirst[s], mcount[s],
                               (const float2 *)(p->tw + p->twoff[s]), p->bank, maxkern[s], st);
    // harmonics of equal fftlen are consecutive rows and consecutive harmonics
    for (int hind = 0; hind < numharm && e == cudaSuccess;) {
        int hend = hind + 1;
        while (hend < numharm && H[hend].fftlen == H[hind].fftlen)
            hend++;
        const int N = H[hind].fftlen;
        const int si = size_index(N);
        const float2 *tw = p->tw + p->twoff[si];
        const int first = (int)H[hind].row0, count = (hend - hind) * kCells;
        e = p_dispatch<PK>(N, (const PolishRow *)p->d_rows, first, count, tw, p->bank, st);
        if (e == cudaSuccess)
            e = p_dispatch<PD>(N, (const PolishHarm *)p->d_harms, hind, hend - hind, tw,
                               (const float2 *)p->windows, p->dfft, st);
        if (e == cudaSuccess)
            e = p_dispatch<PC>(N, (const PolishRow *)p->d_rows, first, count,
                               (const PolishHarm *)p->d_harms, tw, (const float2 *)p->bank,
                               (const float2 *)p->dfft, p->terms, p->tails, st);
        hind = hend;
    }
    if (e == cudaSuccess) {
        ps_argmax_kernel<<<1, kArgThreads, 0, st>>>(p->terms, p->tails, p->d_harms, numharm,
                                                    p->d_best, p->d_bestpow);
        e = cudaGetLastError();
    }
    int best = 0;
    float bpow = 0.0f;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&best, p->d_best, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&bpow, p->d_bestpow, sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return p_cuda(e, "jerk_polish_rzw");
    p->candidates++;

    // ---- the polished values (src/maximize_rzw.c:160-169)
    const int wind = best / (kGrid * kNumR), zind = (best / kNumR) % kGrid, rind = best % kNumR;
    const double nh = numharm;
    *rout = (hhlobin + rind * dr) / nh;
    *zout = ((zin * nh) - kNumWid * kDZ + zind * kDZ / (double)kInterp) / nh;
    *wout = ((win * nh) - kNumWid * kDW + wind * kDW / (double)kInterp) / nh;
    if (maxpow)
        *maxpow = bpow;
    return JERK_OK;
}

// ---------------------------------------------------------------------------
// Complex interpolation at single points: the reference's rzw_interp
// (src/rzwinterp.c:151-228) and rz_interp (src/rzinterp.c:144-235), on
// which its local power (get_localpower3d, src/characteristics.c:75-135)
// and peak derivatives (get_derivs3d, src/characteristics.c:138-191) stand.
// A point correlates 2 khw spectrum bins around floor(r) with the response
// of (frac(r), z, w) at one point per bin: gen_w_response (the cosine series
// and real FFT, as above, with the fractional offset) where |w| >= 1e-4,
// else gen_z_response / gen_r_response.  One CTA per point; the products
// are summed in double and rounded to the float answer.

namespace jerk {
namespace {

struct InterpPoint {
    long long win;  // float2 offset of the staged data window (numkern bins)
    double frac, z, w;
    int numkern;    // 2 kern_half_width
    int npts;       // w responses: the cosine series' length (M = npts / 2)
};

constexpr int kInterpThreads = 256;

template <int NT>
__device__ __forceinline__ void block_sum2(double &a, double &b)
{
    __shared__ double red[2][NT / 32];
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][wid] = a;
        red[1][wid] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        a = 0.0;
        b = 0.0;
        for (int i = 0; i < NT / 32; i++) {
            a += red[0][i];
            b += red[1][i];
        }
    }
}

// the reference's sum for one bin: ans += data x conj(response)
__device__ __forceinline__ void corr_acc(float2 d, float re, float im, double &ar, double &ai)
{
    ar += (double)d.x * re + (double)d.y * im;
    ai += (double)d.y * re - (double)im * d.x;
}

__global__ void __launch_bounds__(kInterpThreads)
    interp_zr_kernel(const InterpPoint *__restrict__ pts, const int *__restrict__ list,
                     const float2 *__restrict__ windows, float2 *__restrict__ ans)
{
    const int pi = list[blockIdx.x];
    const InterpPoint P = pts[pi];
    const float2 *d = windows + P.win;
    const int tid = threadIdx.x, numkern = P.numkern;
    const double z = P.z, roff = P.frac;
    double ar = 0.0, ai = 0.0;
    if (fabs(z) >= 1e-4) {
        // gen_z_response(roff, 1, z, numkern) (src/responses.c:228-313)
        const double absz = fabs(z);
        const double startr0 = roff - 0.5 * z;
        double ipart;
        const double startroffset =
            startr0 < 0.0 ? 1.0 + modf(startr0, &ipart) : modf(startr0, &ipart);
        const int signz = z < 0.0 ? -1 : 1;
        const double zd = signz * 1.4142135623730950488016887242096980785696718753769 / sqrt(absz);
        const double cons = zd / 2.0;
        const double pibyz = M_PI / z;
        const double startr = startr0 + numkern / 2.0;
        for (int ii = tid; ii < numkern; ii += kInterpThreads) {
            const double r = startr - (double)ii;
            const double yy = __dmul_rn(r, zd);
            const double zz = __dadd_rn(yy, __dmul_rn(z, zd));
            const double xx = __dmul_rn(__dmul_rn(pibyz, r), r);
            double sn, cs, fsy, fcy, fsz, fcz;
            sincos(xx, &sn, &cs);
            fresnel(yy, &fsy, &fcy);
            fresnel(zz, &fsz, &fcz);
            const double tmprl = signz * (fcz - fcy);
            const double tmpim = fsy - fsz;
            float re = (float)__dmul_rn(__dsub_rn(__dmul_rn(tmprl, cs), __dmul_rn(tmpim, sn)), cons);
            float im = (float)-__dmul_rn(__dadd_rn(__dmul_rn(tmprl, sn), __dmul_rn(tmpim, cs)), cons);
            if (ii == numkern / 2 && startroffset < 1e-3 && absz < 1e-3) {
                const double z2 = z * z, x2 = startroffset * startroffset;
                double cr = 1.0 - 0.16449340668482264365 * z2;
                double ci = -0.5235987755982988731 * z;
                cr += startroffset * 1.6449340668482264365 * z;
                ci += startroffset * (M_PI - 0.5167712780049970029 * z2);
                cr += x2 * (-6.579736267392905746 + 0.9277056288952613070 * z2);
                ci += x2 * (3.1006276680299820175 * z);
                re = (float)cr;
                im = (float)ci;
            }
            corr_acc(d[ii], re, im, ar, ai);
        }
    } else {
        // gen_r_response(roff, 1, numkern) (src/responses.c:158-226): value ii
        // is exp(i r) sin(r) / r at r = pi (numkern / 2 + roff - ii)
        for (int ii = tid; ii < numkern; ii += kInterpThreads) {
            const double q = numkern / 2.0 + roff - (double)ii;
            float re = 1.0f, im = 0.0f;
            if (q != 0.0) {
                double sn, cs;
                sincospi(q, &sn, &cs);
                const double sinc = sn / (M_PI * q);
                re = (float)(cs * sinc);
                im = (float)(sn * sinc);
            }
            if (ii == numkern / 2 && roff < 1e-3) {
                const double x2 = roff * roff;
                re = (float)(1.0 - 6.579736267392905746 * x2);
                im = (float)(roff * (M_PI - 10.335425560099940058 * x2));
            }
            corr_acc(d[ii], re, im, ar, ai);
        }
    }
    block_sum2<kInterpThreads>(ar, ai);
    if (tid == 0)
        ans[pi] = make_float2((float)ar, (float)ai);
}

// gen_w_response(roff, 1, z, w, numkern) (src/responses.c:333-418): the
// cosine series of npts = 2M samples read as M complex values, FFT'd, and
// the numkern bins around M / 2 split out of the window that the last stage
// drops into shared memory; then the correlation with the data window.
template <int M>
__global__ void __launch_bounds__(FftPlan<M>::T)
    interp_w_kernel(const InterpPoint *__restrict__ pts, const int *__restrict__ list,
                    const float2 *__restrict__ tw, const float2 *__restrict__ windows,
                    float2 *__restrict__ ans)
{
    constexpr int T = FftPlan<M>::T;
    extern __shared__ float2 iw_smem[];
    float2 *buf = iw_smem;
    float2 *win = iw_smem + fft_buf_len<M>();
    const int pi = list[blockIdx.x];
    const InterpPoint P = pts[pi];
    const int tid = threadIdx.x, numkern = P.numkern, npts = P.npts;
    const double z = P.z, w = P.w;
    const double dt = 1.0 / (double)npts;
    const double amp = 2.0 * dt;
    const int fbar = npts / 4;
    const double dfbar = (double)fbar + P.frac;
    const double f = __dadd_rn(__dsub_rn(dfbar, 0.5 * z), w / 12.0);
    const double fd = (z - 0.5 * w) / 2.0;
    const double fdd = w / 6.0;
    auto xval = [&](int n) -> float {
        const double t = __dmul_rn((double)n, dt);
        const double in1 = __dadd_rn(__dmul_rn(t, fdd), fd);
        const double in2 = __dadd_rn(__dmul_rn(t, in1), f);
        const double ph = __dmul_rn(6.2831853071795864769252867665590057683943387987502,
                                    __dmul_rn(t, in2));
        return (float)__dmul_rn(amp, cos(ph));
    };
    auto in = [&](int r) -> float2 {
        const int m = tid + r * T;
        return make_float2(xval(2 * m), xval(2 * m + 1));
    };
    const int lo = M / 2 - numkern / 2;
    auto out = [&](int k, float2 y) {
        if (k >= lo && k <= lo + numkern)
            win[k - lo] = y;
    };
    fft_block<M, -1>(buf, tw, tid, in, out);
    __syncthreads();
    const float2 *d = windows + P.win;
    double ar = 0.0, ai = 0.0;
    for (int k = tid; k < numkern; k += T) {
        const int kc = lo + k;
        const float2 a = win[k], b = win[numkern - k];
        const double hx = 0.5 * ((double)a.x + (double)b.x);
        const double hy = 0.5 * ((double)a.y - (double)b.y);
        const double dx = (double)a.x - (double)b.x;
        const double dy = (double)a.y + (double)b.y;
        double s, c;
        sincospi(-(double)kc / (double)M, &s, &c);
        const double gx = c * dx - s * dy, gy = c * dy + s * dx;
        corr_acc(d[k], (float)(hx + 0.5 * gy), (float)(hy - 0.5 * gx), ar, ai);
    }
    block_sum2<T>(ar, ai);
    if (tid == 0)
        ans[pi] = make_float2((float)ar, (float)ai);
}

template <int M> struct PI {
    static cudaError_t run(const InterpPoint *pts, const int *list, int count, const float2 *tw,
                           const float2 *windows, float2 *ans, int maxkern, cudaStream_t st)
    {
        const int smem = (int)(sizeof(float2) * (fft_buf_len<M>() + maxkern + 1));
        cudaError_t e = cudaFuncSetAttribute(interp_w_kernel<M>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess)
            return e;
        interp_w_kernel<M><<<count, FftPlan<M>::T, smem, st>>>(pts, list, tw, windows, ans);
        return cudaGetLastError();
    }
};

int whw_high(double z, double w) { return w_resp_halfwidth_lowacc(z, w) + 32; }

}  // namespace
}  // namespace jerk

namespace {

// rzw_interp at n points: answers (the reference's float fcomplex) in ans.
int interp_points(jerk_polisher *p, const float2 *data, long long numdata, int n,
                  const double *r, const double *z, const double *w, const int *khw,
                  float2 *ans)
{
    const bool dev = spectrum_on_device(data);
    std::vector<InterpPoint> pts(n);
    std::vector<int> zr, wl[kNumSizes];
    int maxkern[kNumSizes] = {};
    long long win_len = 0;
    std::vector<long long> first(n, 0);
    std::vector<WinSeg> segs;  // a spectrum on the device: the runs to read
    for (int i = 0; i < n; i++) {
        ans[i] = make_float2(0.f, 0.f);
        pts[i].numkern = 0;
        if (r[i] > numdata - 1.0 || r[i] < 0.0)
            continue;  // the reference answers 0 out of range
        double ip;
        const double frac = modf(r[i], &ip);
        const long long intfreq = (long long)ip;
        if (fabs(w[i]) < 1e-4 && fabs(z[i]) < 1e-4) {
            // on a bin: the value itself
            long long b = -1;
            if (frac < 1e-5)
                b = intfreq;
            else if ((1.0 - frac) < 1e-5)
                b = intfreq + 1;
            if (b >= 0) {
                if (dev)
                    segs.push_back(WinSeg{b, i, 1, 1});
                else
                    ans[i] = data[b];
                continue;
            }
        }
        InterpPoint &P = pts[i];
        P.frac = frac;
        P.z = z[i];
        P.w = w[i];
        P.numkern = 2 * khw[i];
        P.win = win_len;
        first[i] = intfreq - khw[i];
        win_len += P.numkern;
        P.npts = 0;
        if (fabs(w[i]) >= 1e-4) {
            P.npts = (int)next2(6 * w_resp_halfwidth_lowacc(z[i], w[i]) + 200 + P.numkern);
            const int M = P.npts / 2;
            const int si = size_index(M);
            if (si < 0 || P.numkern / 2 >= M / 2)
                return p_fail(JERK_EUNSUPPORTED, "rzw_interp: response FFT beyond 8192 points");
            wl[si].push_back(i);
            maxkern[si] = std::max(maxkern[si], P.numkern);
        } else {
            zr.push_back(i);
        }
    }
    std::vector<int> lists(zr);
    int wfirst[kNumSizes], wcount[kNumSizes];
    for (int s = 0; s < kNumSizes; s++) {
        wfirst[s] = (int)lists.size();
        lists.insert(lists.end(), wl[s].begin(), wl[s].end());
        wcount[s] = (int)wl[s].size();
    }
    if (lists.empty() && segs.empty())
        return JERK_OK;
    const size_t nbin = segs.size();  // answers that are bin values
    if (dev)
        for (int i : lists)
            segs.push_back(WinSeg{first[i], pts[i].win, pts[i].numkern, 0});
    // staging: points | lists | windows, or their runs | answers
    const size_t b_pts = sizeof(InterpPoint) * n, b_lists = sizeof(int) * lists.size();
    const size_t o_win = (b_pts + b_lists + 15) & ~(size_t)15;
    const size_t b_win = dev ? sizeof(WinSeg) * segs.size() : sizeof(float2) * win_len;
    const size_t o_ans = (o_win + b_win + 15) & ~(size_t)15, b_ans = sizeof(float2) * n;
    const long long stage = (long long)(o_ans + b_ans);
    cudaError_t e = cudaStreamSynchronize(p->stream);
    if (e == cudaSuccess && stage > p->stage_cap) {
        if (p->h_stage)
            cudaFreeHost(p->h_stage);
        p->h_stage = nullptr;
        p->stage_cap = 0;
        e = cudaMallocHost(&p->h_stage, stage * 2);
        if (e == cudaSuccess)
            p->stage_cap = stage * 2;
    }
    if (e != cudaSuccess)
        return p_cuda(e, "rzw_interp: staging");
    unsigned char *hs = p->h_stage;
    memcpy(hs, pts.data(), b_pts);
    memcpy(hs + b_pts, lists.data(), b_lists);
    float2 *hw = (float2 *)(hs + o_win);
    if (dev)
        memcpy(hw, segs.data(), b_win);
    else
        for (int i = 0; i < n; i++)
            for (int k = 0; k < pts[i].numkern; k++) {
                const long long b = first[i] + k;
                hw[pts[i].win + k] = (b >= 0 && b < numdata) ? data[b] : make_float2(0.f, 0.f);
            }
    // device layout in the polisher's buffers: points in d_rows, lists in
    // d_lists, windows in windows, answers in dfft
    const long long rows_need = (long long)((b_pts + sizeof(PolishRow) - 1) / sizeof(PolishRow));
    if ((e = grow(&p->d_rows, &p->rows_cap, rows_need)) != cudaSuccess ||
        (e = grow(&p->d_lists, &p->lists_cap, (long long)lists.size())) != cudaSuccess ||
        (e = grow(&p->windows, &p->win_cap, std::max(win_len, 1LL))) != cudaSuccess ||
        (e = grow(&p->dfft, &p->dfft_cap, (long long)n)) != cudaSuccess ||
        (dev && (e = grow(&p->d_segs, &p->segs_cap, (long long)segs.size())) != cudaSuccess))
        return p_cuda(e, "rzw_interp: device buffers");
    cudaStream_t st = p->stream;
    const InterpPoint *d_pts = (const InterpPoint *)p->d_rows;
    e = cudaMemcpyAsync(p->d_rows, hs, b_pts, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && b_lists)
        e = cudaMemcpyAsync(p->d_lists, hs + b_pts, b_lists, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && b_win)
        e = cudaMemcpyAsync(dev ? (void *)p->d_segs : (void *)p->windows, hw, b_win,
                            cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && dev) {
        gather_windows_kernel<<<(int)segs.size(), kGatherThreads, 0, st>>>(
            data, numdata, p->d_segs, p->windows, p->dfft);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && !zr.empty()) {
        interp_zr_kernel<<<(int)zr.size(), kInterpThreads, 0, st>>>(d_pts, p->d_lists, p->windows,
                                                                     p->dfft);
        e = cudaGetLastError();
    }
    for (int s = 0; s < kNumSizes && e == cudaSuccess; s++)
        if (wcount[s])
            e = p_dispatch<PI>(kSizes[s], d_pts, (const int *)p->d_lists + wfirst[s], wcount[s],
                               (const float2 *)(p->tw + p->twoff[s]), (const float2 *)p->windows,
                               p->dfft, maxkern[s], st);
    float2 *hans = (float2 *)(hs + o_ans);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(hans, p->dfft, b_ans, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return p_cuda(e, "rzw_interp");
    for (int i = 0; i < n; i++)
        if (pts[i].numkern)
            ans[i] = hans[i];
    for (size_t j = 0; j < nbin; j++)
        ans[segs[j].off] = hans[segs[j].off];
    return JERK_OK;
}

// get_localpower3d's points (src/characteristics.c:95-125): 10 bins either
// side, 5 bins away from r, clamped to the spectrum; freq advances by 1.0.
void localpower_points(double r, long long numdata, std::vector<double> &out)
{
    double lo1 = r - 5 - 10, hi1 = lo1 + 10, lo2 = r + 5, hi2 = lo2 + 10;
    auto clamp = [&](double v) { return v < 0.0 ? 0.0 : (v > (double)numdata ? (double)numdata : v); };
    lo1 = clamp(lo1);
    hi1 = clamp(hi1);
    lo2 = clamp(lo2);
    hi2 = clamp(hi2);
    for (double f = lo1; f < hi1; f += 1.0)
        out.push_back(f);
    for (double f = lo2; f < hi2; f += 1.0)
        out.push_back(f);
}

int local_powers(jerk_polisher *p, const float2 *data, long long numdata, int n, const double *r,
                 const double *z, const double *w, double *out)
{
    std::vector<double> pr, pz, pw;
    std::vector<int> pk, owner;
    for (int i = 0; i < n; i++) {
        std::vector<double> f;
        localpower_points(r[i], numdata, f);
        const int khw = w_resp_halfwidth_lowacc(z[i], w[i]);
        for (double v : f) {
            pr.push_back(v);
            pz.push_back(z[i]);
            pw.push_back(w[i]);
            pk.push_back(khw);
            owner.push_back(i);
        }
    }
    std::vector<float2> a(pr.size());
    if (!pr.empty()) {
        const int rc = interp_points(p, data, numdata, (int)pr.size(), pr.data(), pz.data(),
                                     pw.data(), pk.data(), a.data());
        if (rc != JERK_OK)
            return rc;
    }
    for (int i = 0; i < n; i++)
        out[i] = 0.0;
    for (size_t j = 0; j < pr.size(); j++) {
        const double ar = a[j].x, ai = a[j].y;
        out[owner[j]] += ar * ar + ai * ai;
    }
    for (int i = 0; i < n; i++)
        out[i] /= 20.0;  // NUMLOCPOWAVG
    return JERK_OK;
}

}  // namespace

extern "C" int jerk_local_power(jerk_polisher *p, const void *spectrum, long long numdata, int n,
                                const double *r, const double *z, const double *w, double *out)
{
    if (!p || !spectrum || n < 0 || (n && (!r || !z || !w || !out)))
        return p_fail(JERK_EINVAL, "jerk_local_power: bad argument");
    return local_powers(p, (const float2 *)spectrum, numdata, n, r, z, w, out);
}

extern "C" int jerk_derivs(jerk_polisher *p, const void *spectrum, long long numdata, int n,
                           const double *r, const double *z, const double *w,
                           const double *locpow, jerk_rderivs *out)
{
    if (!p || !spectrum || n < 0 || (n && (!r || !z || !w || !locpow || !out)))
        return p_fail(JERK_EINVAL, "jerk_derivs: bad argument");
    // get_derivs3d (src/characteristics.c:138-191): 5 points 0.003 apart
    // around r at HIGHACC, powers and phases, finite differences
    const double h = 0.003, twoh = 0.006, twohsqrd = 0.000036;
    std::vector<double> pr(5 * (size_t)n), pz(5 * (size_t)n), pw(5 * (size_t)n);
    std::vector<int> pk(5 * (size_t)n);
    for (int i = 0; i < n; i++) {
        const int khw = whw_high(z[i], w[i]);
        double f = r[i] - twoh;
        for (int k = 0; k < 5; k++, f += h) {
            pr[5 * i + k] = f;
            pz[5 * i + k] = z[i];
            pw[5 * i + k] = w[i];
            pk[5 * i + k] = khw;
        }
    }
    std::vector<float2> a(pr.size());
    if (n) {
        const int rc = interp_points(p, (const float2 *)spectrum, numdata, 5 * n, pr.data(),
                                     pz.data(), pw.data(), pk.data(), a.data());
        if (rc != JERK_OK)
            return rc;
    }
    const double twopi = 6.2831853071795864769252867665590057683943387987502;
    for (int i = 0; i < n; i++) {
        double pwr[5], phs[5];
        for (int k = 0; k < 5; k++) {
            const double ar = a[5 * i + k].x, ai = a[5 * i + k].y;
            pwr[k] = ar * ar + ai * ai;
            const double t = atan2(ai, ar);
            phs[k] = t > 0.0 ? t : t + twopi;
        }
        for (int k = 0; k < 4; k++)
            if (fabs(phs[k + 1] - phs[k]) > M_PI)
                phs[k + 1] -= twopi;
        jerk_rderivs &d = out[i];
        d.pow = pwr[2];
        d.phs = phs[2];
        d.dpow = (pwr[3] - pwr[1]) / twoh;
        d.dphs = (phs[3] - phs[1]) / twoh;
        d.d2pow = (pwr[4] - 2.0 * pwr[2] + pwr[0]) / twohsqrd;
        d.d2phs = (phs[4] - 2.0 * phs[2] + phs[0]) / twohsqrd;
        d.locpow = locpow[i];
    }
    return JERK_OK;
}

// The whole default optimisation of one candidate on the GPU, as
// optimize_accelcand runs it with harmonic polishing (src/accel_utils.c:
// 573-657, src/maximize_rzw.c:84-190): local powers, the volume search, then
// for every harmonic the local power and derivatives at the polished point.
extern "C" int jerk_optimize_cand(jerk_polisher *p, const void *spectrum, long long numdata,
                                  int numharm, double rin, double zin, double win,
                                  double *rzw_out, jerk_rderivs *derivs, float *locpow_used)
{
    if (!p || !spectrum || !rzw_out || !derivs || numharm < 1 || numharm > kMaxHarm)
        return p_fail(JERK_EINVAL, "jerk_optimize_cand: bad argument");
    double r[kMaxHarm], z[kMaxHarm], w[kMaxHarm], lp[kMaxHarm];
    for (int i = 0; i < numharm; i++) {
        const int n = numharm - i;
        r[i] = rin * n;
        z[i] = zin * n;
        w[i] = win * n;
    }
    int rc = jerk_local_power(p, spectrum, numdata, numharm, r, z, w, lp);
    if (rc != JERK_OK)
        return rc;
    float lpf[kMaxHarm];
    for (int i = 0; i < numharm; i++)
        lpf[i] = (float)lp[i];
    if (locpow_used)
        memcpy(locpow_used, lpf, sizeof(float) * numharm);
    rc = jerk_polish_rzw(p, spectrum, numdata, numharm, rin, zin, win, lpf, &rzw_out[0],
                         &rzw_out[1], &rzw_out[2], nullptr);
    if (rc != JERK_OK)
        return rc;
    for (int i = 0; i < numharm; i++) {
        const int hh = i + 1;
        r[i] = rzw_out[0] * hh;
        z[i] = rzw_out[1] * hh;
        w[i] = rzw_out[2] * hh;
    }
    rc = jerk_local_power(p, spectrum, numdata, numharm, r, z, w, lp);
    if (rc != JERK_OK)
        return rc;
    for (int i = 0; i < numharm; i++)
        lp[i] = (double)(float)lp[i];  // a float there, as the reference holds it
    return jerk_derivs(p, spectrum, numdata, numharm, r, z, w, lp, derivs);
}
