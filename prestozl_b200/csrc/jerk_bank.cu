// Kernel-bank generation on the GPU.
//
// The reference builds, for every subharmonic and every (w, z) of its grid,
// the Fourier response of a signal with f-dot z and f-dot-dot w, places it
// wrapped around an fftlen array and takes its forward FFT -- on the host,
// in double precision plus float FFTW (src/accel_utils.c:151-168
// init_kernel, src/responses.c:158-418 gen_r/z/w_response,
// src/corr_prep.c:92-114 place_complex_kernel).  Here every kernel is one
// CTA, in two passes:
//
//   bank_response_kernel   the numkern response values in double, rounded to
//                          float and placed into the bank row (zeros between):
//     w != 0  the reference's method: a float cosine series of num_pts
//             samples, zero-padded to twice its length, whose real FFT is
//             sampled at numkern bins; here those bins are evaluated as a
//             direct DFT in double (phasor recurrence, re-seeded every 64
//             samples), which is the same sum without the FFT's rounding;
//     w == 0, z != 0  the closed form with Fresnel integrals;
//     w == 0, z == 0  the interbinning sinc.
//   bank_fft_kernel<N>     in-place forward FFT (sign -1) of each row with the
//                          shared-memory Stockham FFT of jerk_fft.cuh.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include "jerk.h"
#include "jerk_fft.cuh"
#include "jerk_kernels.cuh"
#include "jerk_resp.cuh"

namespace jerk {


constexpr int kBankThreads = 256;


__global__ void __launch_bounds__(kBankThreads)
    bank_response_kernel(const BankRow *rows, float2 *bank)
{
    extern __shared__ float xs[];
    const BankRow R = rows[blockIdx.x];
    const int tid = threadIdx.x;
    float2 *row = bank + R.off;
    const int numkern = R.numkern;
    const int numbetween = 2;

    // zero the parts of the row the response does not cover
    for (int m = numkern / 2 + tid; m < R.fftlen - numkern / 2; m += kBankThreads)
        row[m] = make_float2(0.f, 0.f);

    const double z = R.z, w = R.w;
    if (fabs(w) >= 1e-4) {
        // gen_w_response (src/responses.c:333-418), roffset = 0
        const int npts = R.num_pts;
        const double dt = 1.0 / (double)npts;
        const double amp = 2.0 * dt;
        const int fbar = npts / 4;
        const double f = __dadd_rn(__dsub_rn((double)fbar, 0.5 * z), w / 12.0);
        const double fd = (z - 0.5 * w) / 2.0;
        const double fdd = w / 6.0;
        for (int n = tid; n < npts; n += kBankThreads) {
            const double t = __dmul_rn((double)n, dt);
            // TWOPI * (t * (t * (t * fdd + fd) + f)), no contraction
            const double in1 = __dadd_rn(__dmul_rn(t, fdd), fd);
            const double in2 = __dadd_rn(__dmul_rn(t, in1), f);
            const double ph = __dmul_rn(6.2831853071795864769252867665590057683943387987502,
                                        __dmul_rn(t, in2));
            xs[n] = (float)__dmul_rn(amp, cos(ph));
        }
        __syncthreads();
        // complex bins k0 + k of the length-2*npts real DFT
        const int L = npts * numbetween;
        const int k0 = fbar * numbetween - numkern / 2;
        for (int k = tid; k < numkern; k += kBankThreads) {
            const long long kc = k0 + k;
            double accr = 0.0, acci = 0.0;
            double wr, wi;  // exp(-2 pi i kc / L)
            sincospi(-2.0 * (double)kc / (double)L, &wi, &wr);
            for (int n0 = 0; n0 < npts; n0 += 64) {
                double pr, pi;  // exp(-2 pi i kc n0 / L), exact reduction of kc*n0 mod L
                const long long m = (kc * (long long)n0) % L;
                sincospi(-2.0 * (double)m / (double)L, &pi, &pr);
                const int nend = min(npts, n0 + 64);
                for (int n = n0; n < nend; n++) {
                    const double x = (double)xs[n];
                    accr = fma(x, pr, accr);
                    acci = fma(x, pi, acci);
                    const double tr = pr * wr - pi * wi;
                    pi = pr * wi + pi * wr;
                    pr = tr;
                }
            }
            row[placed(k, numkern, R.fftlen)] = make_float2((float)accr, (float)acci);
        }
    } else if (fabs(z) >= 1e-4) {
        // gen_z_response (src/responses.c:228-313), roffset = 0
        const double absz = fabs(z);
        const double startr0 = -0.5 * z;
        const int signz = z < 0.0 ? -1 : 1;
        const double zd = signz * 1.4142135623730950488016887242096980785696718753769 / sqrt(absz);
        const double cons = zd / 2.0;
        const double pibyz = M_PI / z;
        const double startr = startr0 + numkern / (double)(2 * numbetween);
        const double delta = -1.0 / numbetween;
        for (int ii = tid; ii < numkern; ii += kBankThreads) {
            const double r = startr + ii * delta;
            const double yy = __dmul_rn(r, zd);
            const double zz = __dadd_rn(yy, __dmul_rn(z, zd));
            const double xx = __dmul_rn(__dmul_rn(pibyz, r), r);
            double sn, cs, fsy, fcy, fsz, fcz;
            sincos(xx, &sn, &cs);
            fresnel(yy, &fsy, &fcy);
            fresnel(zz, &fsz, &fcz);
            const double tmprl = signz * (fcz - fcy);
            const double tmpim = fsy - fsz;
            const float re = (float)__dmul_rn(__dsub_rn(__dmul_rn(tmprl, cs), __dmul_rn(tmpim, sn)), cons);
            const float im = (float)-__dmul_rn(__dadd_rn(__dmul_rn(tmprl, sn), __dmul_rn(tmpim, cs)), cons);
            row[placed(ii, numkern, R.fftlen)] = make_float2(re, im);
        }
    } else {
        // gen_r_response (src/responses.c:158-226), roffset = 0:
        // value ii = exp(i r) sin(r) / r at r = pi (numkern/4 - ii/2)
        for (int ii = tid; ii < numkern; ii += kBankThreads) {
            const double q = numkern / (double)(2 * numbetween) - 0.5 * ii;  // r / pi
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

struct BankGroup {
    int first, count;  // rows [first, first + count) of one fftlen
};

// Twiddle tables beside the buffer in shared memory, except where they do not
// fit (15360): read from global memory there.
template <int N>
struct BankTwInSmem {
    static constexpr bool value =
        (size_t)(fft_buf_len<N>() + FftPlan<N>::twsize()) * 8 <= 200 * 1024;
};

template <int N>
__global__ void __launch_bounds__(FftPlan<N>::T)
    bank_fft_kernel(const BankRow *rows, int first, const float2 *twiddles, int twoff,
                    float2 *bank)
{
    constexpr int R0 = FftPlan<N>::R0;
    constexpr int T = FftPlan<N>::T;
    constexpr int TWN = FftPlan<N>::twsize();
    extern __shared__ float2 smb[];
    float2 *buf = smb;
    const float2 *tw = BankTwInSmem<N>::value ? smb + fft_buf_len<N>() : twiddles + twoff;
    const int tid = threadIdx.x;
    const BankRow R = rows[first + blockIdx.x];
    float2 *row = bank + R.off;
    if constexpr (BankTwInSmem<N>::value) {
        for (int i = tid; i < TWN; i += T)
            smb[fft_buf_len<N>() + i] = twiddles[twoff + i];
    }
    __syncthreads();
    auto in = [&](int r) -> float2 { return row[tid + r * (N / R0)]; };
    auto out = [&](int m, float2 y) { row[m] = y; };
    fft_block<N, -1>(buf, tw, tid, in, out);
}

template <int N>
static cudaError_t launch_bank_fft(const BankRow *rows, int first, int count, const float2 *tw,
                                   int twoff, float2 *bank, cudaStream_t st)
{
    const size_t smem =
        sizeof(float2) * (fft_buf_len<N>() + (BankTwInSmem<N>::value ? FftPlan<N>::twsize() : 0));
    cudaError_t e = cudaFuncSetAttribute(bank_fft_kernel<N>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    bank_fft_kernel<N><<<count, FftPlan<N>::T, smem, st>>>(rows, first, tw, twoff, bank);
    return cudaGetLastError();
}

cudaError_t launch_bank_fft_any(int N, const BankRow *rows, int first, int count, const float2 *tw,
                                int twoff, float2 *bank, cudaStream_t st)
{
    switch (N) {
    case 128: return launch_bank_fft<128>(rows, first, count, tw, twoff, bank, st);
    case 192: return launch_bank_fft<192>(rows, first, count, tw, twoff, bank, st);
    case 256: return launch_bank_fft<256>(rows, first, count, tw, twoff, bank, st);
    case 384: return launch_bank_fft<384>(rows, first, count, tw, twoff, bank, st);
    case 512: return launch_bank_fft<512>(rows, first, count, tw, twoff, bank, st);
    case 768: return launch_bank_fft<768>(rows, first, count, tw, twoff, bank, st);
    case 1024: return launch_bank_fft<1024>(rows, first, count, tw, twoff, bank, st);
    case 1280: return launch_bank_fft<1280>(rows, first, count, tw, twoff, bank, st);
    case 2048: return launch_bank_fft<2048>(rows, first, count, tw, twoff, bank, st);
    case 4096: return launch_bank_fft<4096>(rows, first, count, tw, twoff, bank, st);
    case 5120: return launch_bank_fft<5120>(rows, first, count, tw, twoff, bank, st);
    case 7680: return launch_bank_fft<7680>(rows, first, count, tw, twoff, bank, st);
    case 8192: return launch_bank_fft<8192>(rows, first, count, tw, twoff, bank, st);
    case 10240: return launch_bank_fft<10240>(rows, first, count, tw, twoff, bank, st);
    case 15360: return launch_bank_fft<15360>(rows, first, count, tw, twoff, bank, st);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_bank_response(const BankRow *rows, int nrows, int max_pts, float2 *bank,
                                 cudaStream_t st)
{
    const size_t smem = sizeof(float) * (size_t)(max_pts > 0 ? max_pts : 1);
    cudaError_t e = cudaFuncSetAttribute(bank_response_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    bank_response_kernel<<<nrows, kBankThreads, smem, st>>>(rows, bank);
    return cudaGetLastError();
}

}  // namespace jerk
