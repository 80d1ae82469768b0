// Subband dedispersion on the GPU: the two steps prepsubband_cu runs on
// every block of subband data before the DM trials go to the search
// (src/prepsubband_cu.c:1140-1165):
//
//   jerk_downsample_subbands  DownsampDataArray (src/prepsubband_kernels.cu:
//                             23-46; the CPU form src/prepsubband.c:984-1001):
//                             ds[t][s] = (sum over k < bs of in[t bs + k][s]) / bs
//   jerk_dedisp_subbands      getDedisp (src/prepsubband_kernels.cu:48-74; the
//                             CPU form float_dedisp, src/dispersion.c:208-231):
//                             out[dm][t] = sum over s of x[t + off[dm][s]][s],
//                             x = last ++ cur, the previous and the current
//                             block of worklen samples of nsub subbands
//
// Both sum in the reference's order (k, then s ascending) in FP32, so the
// results are bit-exact with the reference's.
//
// The reference's getDedisp runs one thread per (dm, t) and makes nsub
// global loads each nsub floats apart.  Here one CTA takes a tile of T
// samples for a group of G consecutive DMs: for every subband s it stages
// the window of x that the group's DMs read -- T + (largest - smallest
// offset of s in the group) samples -- into shared memory once, transposed
// to [s][t] so that a warp's reads are consecutive words, and every staged
// value serves all G DMs.  Windows of four subbands come in as one 16-byte
// load per sample when nsub is a multiple of 4.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <vector>

#include "jerk.h"
#include "jerk_kernels.cuh"

using jerk::set_error;

namespace {

constexpr int kDdThreads = 256;
constexpr int kDsThreads = 256;
constexpr size_t kSmemPreferred = 100 * 1024;  // two CTAs per SM
constexpr size_t kSmemMax = 227 * 1024;

// V: subbands per window load (4: one 16-byte load per sample; 1: one);
// KT: outputs per thread per pass, T / KT apart.
template <int V, int KT>
__global__ void __launch_bounds__(kDdThreads)
dedisp_kernel(const float *__restrict__ cur, const float *__restrict__ last,
              float *__restrict__ out, const int *__restrict__ offsets,
              const int *__restrict__ glo, const int *__restrict__ gbase, int worklen, int nsub,
              int numdms, int G, int T)
{
    extern __shared__ float sm[];
    const int g = blockIdx.y;
    const int t0 = blockIdx.x * T;
    const int d0 = g * G;
    const int gd = min(G, numdms - d0);
    const int *lo_g = glo + (size_t)g * nsub;
    const int *base_g = gbase + (size_t)g * (nsub + 1);
    const int total = base_g[nsub];
    float *win = sm;                             // [s][T + span_s], rows at base[s]
    int *pos = (int *)(sm + ((total + 3) & ~3));  // [d][s]: row base + offset - lowest offset
    int *lo = pos + G * nsub;         // [s]: the group's lowest offset
    int *base = lo + nsub;            // [s + 1]
    for (int i = threadIdx.x; i < nsub; i += kDdThreads)
        lo[i] = lo_g[i];
    for (int i = threadIdx.x; i <= nsub; i += kDdThreads)
        base[i] = base_g[i];
    __syncthreads();
    for (int i = threadIdx.x; i < gd * nsub; i += kDdThreads) {
        const int d = i / nsub, s = i - d * nsub;
        pos[i] = base[s] + offsets[(size_t)(d0 + d) * nsub + s] - lo[s];
    }
    // x[tau] = last[tau] for tau < worklen, cur[tau - worklen] after
    const long long tau_end = 2LL * worklen;
    // (the window stores share the array with lo and base, so the loops
    // below keep what they need of those in registers)
    if (V == 4) {
        for (int q = 0; q < nsub / 4; q++) {
            int slo[4], sw[4], sb[4];
            int qlo = INT_MAX, qend = INT_MIN;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int s = 4 * q + j;
                slo[j] = lo[s];
                sb[j] = base[s];
                sw[j] = base[s + 1] - sb[j];
                qlo = min(qlo, slo[j]);
                qend = max(qend, slo[j] + sw[j]);
            }
            for (int i = threadIdx.x; i < qend - qlo; i += kDdThreads) {
                const long long tau = (long long)t0 + qlo + i;
                float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                if (tau < tau_end) {
                    const float *src = tau < worklen ? last + tau * nsub
                                                     : cur + (tau - worklen) * nsub;
                    v = __ldg((const float4 *)(src + 4 * q));
                }
                const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int p = qlo + i - slo[j];
                    if (p >= 0 && p < sw[j])
                        win[sb[j] + p] = vv[j];
                }
            }
        }
    } else {
        for (int s = 0; s < nsub; s++) {
            const int b = base[s], W = base[s + 1] - b;
            const long long tau0 = (long long)t0 + lo[s];
            for (int i = threadIdx.x; i < W; i += kDdThreads) {
                const long long tau = tau0 + i;
                float v = 0.f;
                if (tau < tau_end)
                    v = tau < worklen ? __ldg(last + tau * nsub + s)
                                      : __ldg(cur + (tau - worklen) * nsub + s);
                win[b + i] = v;
            }
        }
    }
    __syncthreads();
    // float_dedisp starts each sum at -approx_mean = -0.0f and adds the
    // subbands in ascending order
    const int TQ = T / KT;
    for (int it = threadIdx.x; it < gd * TQ; it += kDdThreads) {
        const int d = it / TQ, tq = it - d * TQ;
        const int *pd = pos + d * nsub;
        float v[KT];
#pragma unroll
        for (int k = 0; k < KT; k++)
            v[k] = -0.0f;
        int s = 0;
        if (V == 4)  // rows of pos start on 16 bytes: four positions per load
            for (; s < nsub; s += 4) {
                const int4 p4 = *(const int4 *)(pd + s);
                const int pp[4] = {p4.x, p4.y, p4.z, p4.w};
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const float *w = win + pp[j] + tq;
#pragma unroll
                    for (int k = 0; k < KT; k++)
                        v[k] += w[k * TQ];
                }
            }
        for (; s < nsub; s++) {
            const float *w = win + pd[s] + tq;
#pragma unroll
            for (int k = 0; k < KT; k++)
                v[k] += w[k * TQ];
        }
        float *o = out + (size_t)(d0 + d) * worklen + t0;
#pragma unroll
        for (int k = 0; k < KT; k++) {
            const int t = tq + k * TQ;
            if (t0 + t < worklen)
                o[t] = v[k];
        }
    }
}

__global__ void __launch_bounds__(kDsThreads)
downsample_kernel(float *__restrict__ out, const float *__restrict__ in, long long n, int bs,
                  int nsub)
{
    for (long long i = blockIdx.x * (long long)kDsThreads + threadIdx.x; i < n;
         i += (long long)gridDim.x * kDsThreads) {
        const long long t = i / nsub;
        const int s = (int)(i - t * nsub);
        const float *p = in + t * bs * nsub + s;
        float v = 0.0f;
        for (int k = 0; k < bs; k++)
            v += __ldg(p + (long long)k * nsub);
        out[i] = v / (float)bs;
    }
}

int num_sms()
{
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            sms < 1)
            sms = 148;
    }
    return sms;
}

int dd_cuda(cudaError_t e, const char *what)
{
    static thread_local char buf[256];
    snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    return set_error(JERK_ECUDA, buf);
}

}  // namespace

struct jerk_dedisperser {
    int worklen = 0, nsub = 0, numdms = 0, G = 1, T = 32, ngroups = 0;
    size_t smem = 0;
    int *d_offsets = nullptr, *d_glo = nullptr, *d_gbase = nullptr;
    std::vector<int> h_offsets;
};

namespace {

// Per group of G DMs and subband s: the lowest offset and the window rows'
// bases; returns the largest shared-memory footprint over the groups.
size_t dd_tables(const int *off, int numdms, int nsub, int G, int T, std::vector<int> *lo,
                 std::vector<int> *base)
{
    const int ngroups = (numdms + G - 1) / G;
    if (lo) {
        lo->assign((size_t)ngroups * nsub, 0);
        base->assign((size_t)ngroups * (nsub + 1), 0);
    }
    size_t worst = 0;
    for (int g = 0; g < ngroups; g++) {
        long long total = 0;
        for (int s = 0; s < nsub; s++) {
            int mn = INT_MAX, mx = INT_MIN;
            for (int d = g * G; d < std::min(numdms, (g + 1) * G); d++) {
                mn = std::min(mn, off[(size_t)d * nsub + s]);
                mx = std::max(mx, off[(size_t)d * nsub + s]);
            }
            if (lo) {
                (*lo)[(size_t)g * nsub + s] = mn;
                (*base)[(size_t)g * (nsub + 1) + s] = (int)total;
            }
            total += T + (mx - mn);
        }
        if (lo)
            (*base)[(size_t)g * (nsub + 1) + nsub] = (int)total;
        const size_t bytes = sizeof(float) * (size_t)((total + 3) & ~3LL) +
                             sizeof(int) * ((size_t)G * nsub + 2 * nsub + 1);
        worst = std::max(worst, bytes);
    }
    return worst;
}

// The offsets table on the host: copied from device memory (as getDedisp
// receives it) when it lives there.
int host_offsets(const int *offsets, long long n, std::vector<int> &buf, const int **out)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, offsets) != cudaSuccess) {
        cudaGetLastError();
        *out = offsets;
        return JERK_OK;
    }
    if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) {
        *out = offsets;
        return JERK_OK;
    }
    buf.resize((size_t)n);
    const cudaError_t e = cudaMemcpy(buf.data(), offsets, sizeof(int) * n, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return dd_cuda(e, "dedisperser offsets");
    *out = buf.data();
    return JERK_OK;
}

}  // namespace

// Host only: checks the sizes and a host offsets table and chooses the
// tiling -- the widest tile (256, 128), then the largest DM group, whose
// shared memory fits two CTAs per SM; else tiles of 64 or 32 samples with up
// to 227 KB.
extern "C" int jerk_dedisp_plan(int worklen, int nsub, int numdms, const int *offsets,
                                int *group_dms, int *tile_samples, long long *smem_bytes)
{
    if (!offsets)
        return set_error(JERK_EINVAL, "jerk_dedisp_plan: null pointer");
    if (worklen < 1 || nsub < 1 || numdms < 1)
        return set_error(JERK_EINVAL, "jerk_dedisp_plan: worklen, nsub, numdms must be > 0");
    if ((long long)worklen * nsub * 2 >= (1LL << 40) || (long long)numdms * nsub > INT_MAX)
        return set_error(JERK_EINVAL, "jerk_dedisp_plan: sizes too large");
    for (long long i = 0; i < (long long)numdms * nsub; i++)
        if (offsets[i] < 0 || offsets[i] > worklen)
            return set_error(JERK_EINVAL, "jerk_dedisp_plan: every offset must lie in [0, worklen]");
    int G = 0, T = 0;
    size_t smem = 0;
    for (int t : {256, 128, 64, 32}) {
        const size_t cap = t >= 128 ? kSmemPreferred : kSmemMax;
        for (int gsz : {32, 16, 8, 4, 2, 1}) {
            const size_t b = dd_tables(offsets, numdms, nsub, gsz, t, nullptr, nullptr);
            if (b <= cap) {
                G = gsz;
                T = t;
                smem = b;
                break;
            }
        }
        if (G)
            break;
    }
    if (!G)
        return set_error(JERK_EUNSUPPORTED,
                         "jerk_dedisp_plan: a subband window does not fit in shared memory");
    if ((numdms + G - 1) / G > 65535)
        return set_error(JERK_EUNSUPPORTED, "jerk_dedisp_plan: too many DM groups");
    if (group_dms)
        *group_dms = G;
    if (tile_samples)
        *tile_samples = T;
    if (smem_bytes)
        *smem_bytes = (long long)smem;
    return JERK_OK;
}

extern "C" int jerk_dedisperser_create(jerk_dedisperser **out, int worklen, int nsub, int numdms,
                                       const int *offsets_in)
{
    if (!out || !offsets_in)
        return set_error(JERK_EINVAL, "jerk_dedisperser_create: null pointer");
    *out = nullptr;
    if (worklen < 1 || nsub < 1 || numdms < 1 || (long long)numdms * nsub > INT_MAX)
        return set_error(JERK_EINVAL, "jerk_dedisperser_create: bad sizes");
    std::vector<int> hbuf;
    const int *offsets = nullptr;
    int rc = host_offsets(offsets_in, (long long)numdms * nsub, hbuf, &offsets);
    if (rc != JERK_OK)
        return rc;
    int G = 0, T = 0;
    if ((rc = jerk_dedisp_plan(worklen, nsub, numdms, offsets, &G, &T, nullptr)) != JERK_OK)
        return rc;
    jerk_dedisperser *d = new jerk_dedisperser;
    d->worklen = worklen;
    d->nsub = nsub;
    d->numdms = numdms;
    d->G = G;
    d->T = T;
    d->ngroups = (numdms + G - 1) / G;
    std::vector<int> lo, base;
    d->smem = dd_tables(offsets, numdms, nsub, G, T, &lo, &base);
    d->h_offsets.assign(offsets, offsets + (size_t)numdms * nsub);
    const size_t b_off = sizeof(int) * (size_t)numdms * nsub;
    cudaError_t e = cudaMalloc(&d->d_offsets, b_off);
    if (e == cudaSuccess)
        e = cudaMalloc(&d->d_glo, sizeof(int) * lo.size());
    if (e == cudaSuccess)
        e = cudaMalloc(&d->d_gbase, sizeof(int) * base.size());
    if (e == cudaSuccess)
        e = cudaMemcpy(d->d_offsets, offsets, b_off, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(d->d_glo, lo.data(), sizeof(int) * lo.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(d->d_gbase, base.data(), sizeof(int) * base.size(), cudaMemcpyHostToDevice);
    for (auto k : {dedisp_kernel<4, 8>, dedisp_kernel<4, 4>, dedisp_kernel<1, 8>,
                   dedisp_kernel<1, 4>})
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)kSmemMax);
    if (e != cudaSuccess) {
        jerk_dedisperser_destroy(d);
        return dd_cuda(e, "jerk_dedisperser_create");
    }
    *out = d;
    return JERK_OK;
}

extern "C" void jerk_dedisperser_destroy(jerk_dedisperser *d)
{
    if (!d)
        return;
    cudaFree(d->d_offsets);
    cudaFree(d->d_glo);
    cudaFree(d->d_gbase);
    delete d;
}

extern "C" int jerk_dedisperser_shape(const jerk_dedisperser *d, int *group_dms, int *tile_samples)
{
    if (!d)
        return set_error(JERK_EINVAL, "jerk_dedisperser_shape: null pointer");
    if (group_dms)
        *group_dms = d->G;
    if (tile_samples)
        *tile_samples = d->T;
    return JERK_OK;
}

extern "C" int jerk_dedisperser_matches(const jerk_dedisperser *d, int worklen, int nsub,
                                        int numdms, const int *offsets_in)
{
    if (!d || !offsets_in || d->worklen != worklen || d->nsub != nsub || d->numdms != numdms)
        return 0;
    std::vector<int> hbuf;
    const int *offsets = nullptr;
    if (host_offsets(offsets_in, (long long)numdms * nsub, hbuf, &offsets) != JERK_OK)
        return 0;
    return std::equal(d->h_offsets.begin(), d->h_offsets.end(), offsets) ? 1 : 0;
}

extern "C" int jerk_dedisp_subbands(jerk_dedisperser *d, const float *cur, const float *last,
                                    float *out, void *stream)
{
    if (!d || !cur || !last || !out)
        return set_error(JERK_EINVAL, "jerk_dedisp_subbands: null pointer");
    cudaStream_t st = (cudaStream_t)stream;
    const dim3 grid((d->worklen + d->T - 1) / d->T, d->ngroups);
    const bool quads = d->nsub % 4 == 0 && ((uintptr_t)cur % 16) == 0 && ((uintptr_t)last % 16) == 0;
    // 8 outputs per thread on 256-sample tiles (a warp per DM row), else 4
    auto kern = quads ? (d->T >= 256 ? dedisp_kernel<4, 8> : dedisp_kernel<4, 4>)
                      : (d->T >= 256 ? dedisp_kernel<1, 8> : dedisp_kernel<1, 4>);
    kern<<<grid, kDdThreads, d->smem, st>>>(cur, last, out, d->d_offsets, d->d_glo, d->d_gbase,
                                            d->worklen, d->nsub, d->numdms, d->G, d->T);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? JERK_OK : dd_cuda(e, "jerk_dedisp_subbands");
}

extern "C" int jerk_downsample_subbands(float *out, const float *in, int worklen, int bs, int nsub,
                                        void *stream)
{
    if (!out || !in)
        return set_error(JERK_EINVAL, "jerk_downsample_subbands: null pointer");
    if (worklen < 1 || bs < 1 || nsub < 1)
        return set_error(JERK_EINVAL, "jerk_downsample_subbands: worklen, bs, nsub must be > 0");
    const long long n = (long long)worklen * nsub;
    const long long blocks = std::min<long long>((n + kDsThreads - 1) / kDsThreads, 8LL * num_sms());
    downsample_kernel<<<(int)blocks, kDsThreads, 0, (cudaStream_t)stream>>>(out, in, n, bs, nsub);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? JERK_OK : dd_cuda(e, "jerk_downsample_subbands");
}
