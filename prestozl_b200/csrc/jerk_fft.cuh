// Shared-memory mixed-radix Stockham FFT for one CTA (sm_100a, FP32).
//
// One CTA of T threads transforms one N-point complex sequence.  The first
// stage takes its inputs from a functor (so the caller can fuse a load and a
// multiply into it, and keep per-thread operands such as a kernel row in
// registers across many transforms), the middle stages run in place in a
// shared buffer of N float2, and the last stage hands every output to a
// second functor (so the caller can fuse |.|^2 and the store into it).
//
// Stage s with radix R and Ns = product of the earlier radices (Stockham
// autosort, decimation in time):
//   butterfly j in [0, N/R):  v[r] = x[j + r*N/R] * W^(r * (j % Ns) * N/(Ns*R))
//                             y = DFT_R(v)
//                             out[(j/Ns)*Ns*R + j%Ns + r*Ns] = y[r]
// with W = exp(SIGN * 2*pi*i / N).  Twiddles come from a table of the N
// forward roots exp(-2*pi*i*m/N) (computed in double on the host), conjugated
// for SIGN = +1.
#pragma once

#include <cuda_runtime.h>

namespace jerk {

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b): the correlation product of the reference, (ar*br + ai*bi, ai*br - ar*bi)
__device__ __forceinline__ float2 cmulconj(float2 a, float2 b)
{
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by SIGN * i
template <int SIGN>
__device__ __forceinline__ float2 mul_si(float2 a)
{
    return SIGN > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// In-register DFT of radix R with exponent sign SIGN (unnormalised).
template <int R, int SIGN> struct Dft;

template <int SIGN> struct Dft<2, SIGN> {
    __device__ __forceinline__ static void run(float2 *v)
    {
        float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <int SIGN> struct Dft<4, SIGN> {
    __device__ __forceinline__ static void run(float2 *v)
    {
        float2 a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
        float2 c = cadd(v[1], v[3]), d = mul_si<SIGN>(csub(v[1], v[3]));
        v[0] = cadd(a, c);
        v[1] = cadd(b, d);
        v[2] = csub(a, c);
        v[3] = csub(b, d);
    }
};

template <int SIGN> struct Dft<8, SIGN> {
    __device__ __forceinline__ static void run(float2 *v)
    {
        float2 e[4] = {v[0], v[2], v[4], v[6]};
        float2 o[4] = {v[1], v[3], v[5], v[7]};
        Dft<4, SIGN>::run(e);
        Dft<4, SIGN>::run(o);
        const float h = 0.70710678118654752440f;
        // W8^1 = h(1 + SIGN i), W8^2 = SIGN i, W8^3 = h(-1 + SIGN i)
        float2 o1 = make_float2(h * (o[1].x - SIGN * o[1].y), h * (o[1].y + SIGN * o[1].x));
        float2 o2 = mul_si<SIGN>(o[2]);
        float2 o3 = make_float2(h * (-o[3].x - SIGN * o[3].y), h * (-o[3].y + SIGN * o[3].x));
        v[0] = cadd(e[0], o[0]);
        v[4] = csub(e[0], o[0]);
        v[1] = cadd(e[1], o1);
        v[5] = csub(e[1], o1);
        v[2] = cadd(e[2], o2);
        v[6] = csub(e[2], o2);
        v[3] = cadd(e[3], o3);
        v[7] = csub(e[3], o3);
    }
};

// 16 = 4 x 4: DFT4 over n1 for each n2, twiddle W16^(n2 k1), DFT4 over n2.
template <int SIGN> struct Dft<16, SIGN> {
    __device__ __forceinline__ static float2 w16(float2 a, int m)
    {
        const float c1 = 0.92387953251128675613f;  // cos(pi/8)
        const float s1 = 0.38268343236508977173f;  // sin(pi/8)
        const float h = 0.70710678118654752440f;
        switch (m) {
        case 0: return a;
        case 1: return cmul(a, make_float2(c1, SIGN * s1));
        case 2: return make_float2(h * (a.x - SIGN * a.y), h * (a.y + SIGN * a.x));
        case 3: return cmul(a, make_float2(s1, SIGN * c1));
        case 4: return mul_si<SIGN>(a);
        case 6: return make_float2(h * (-a.x - SIGN * a.y), h * (-a.y + SIGN * a.x));
        case 9: return cmul(a, make_float2(-c1, -SIGN * s1));
        default: return a;  // unreachable for n2, k1 in [0, 4)
        }
    }
    __device__ __forceinline__ static void run(float2 *v)
    {
        float2 a[4][4];
#pragma unroll
        for (int n2 = 0; n2 < 4; n2++) {
            float2 t[4] = {v[n2], v[n2 + 4], v[n2 + 8], v[n2 + 12]};
            Dft<4, SIGN>::run(t);
#pragma unroll
            for (int k1 = 0; k1 < 4; k1++)
                a[n2][k1] = w16(t[k1], n2 * k1);
        }
#pragma unroll
        for (int k1 = 0; k1 < 4; k1++) {
            float2 t[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
            Dft<4, SIGN>::run(t);
#pragma unroll
            for (int k2 = 0; k2 < 4; k2++)
                v[k1 + 4 * k2] = t[k2];
        }
    }
};

template <int SIGN> struct Dft<3, SIGN> {
    __device__ __forceinline__ static void run(float2 *v)
    {
        const float s3 = 0.86602540378443864676f;  // sin(2 pi / 3)
        float2 t = cadd(v[1], v[2]);
        float2 d = mul_si<SIGN>(cscale(csub(v[1], v[2]), s3));
        float2 m = make_float2(v[0].x - 0.5f * t.x, v[0].y - 0.5f * t.y);
        v[0] = cadd(v[0], t);
        v[1] = cadd(m, d);
        v[2] = csub(m, d);
    }
};

template <int SIGN> struct Dft<5, SIGN> {
    __device__ __forceinline__ static void run(float2 *v)
    {
        const float c1 = 0.30901699437494742410f;   // cos(2 pi/5)
        const float c2 = -0.80901699437494742410f;  // cos(4 pi/5)
        const float s1 = 0.95105651629515357212f;   // sin(2 pi/5)
        const float s2 = 0.58778525229247312917f;   // sin(4 pi/5)
        float2 a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
        float2 a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
        float2 x0 = v[0];
        float2 p1 = make_float2(x0.x + c1 * a1.x + c2 * a2.x, x0.y + c1 * a1.y + c2 * a2.y);
        float2 p2 = make_float2(x0.x + c2 * a1.x + c1 * a2.x, x0.y + c2 * a1.y + c1 * a2.y);
        float2 q1 = mul_si<SIGN>(make_float2(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y));
        float2 q2 = mul_si<SIGN>(make_float2(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y));
        v[0] = make_float2(x0.x + a1.x + a2.x, x0.y + a1.y + a2.y);
        v[1] = cadd(p1, q1);
        v[4] = csub(p1, q1);
        v[2] = cadd(p2, q2);
        v[3] = csub(p2, q2);
    }
};

// Radix plans: the first radix fixes the thread count T = N / R0.
//
// Twiddles live in per-stage tables: stage s >= 1 (Ns = product of the
// earlier radices, radix R) has Ns * R entries W_{Ns R}^(r k) at [r * Ns + k],
// so the lanes of a warp (consecutive k = j % Ns) read consecutive entries.
template <int N> struct FftPlan;
#define JERK_FFT_PLAN(NN, ...)                                                  \
    template <> struct FftPlan<NN> {                                            \
        static constexpr int radices[] = {__VA_ARGS__};                         \
        static constexpr int nstages = sizeof(radices) / sizeof(int);           \
        static constexpr int R0 = radices[0];                                   \
        static constexpr int T = NN / R0;                                       \
        /* offset of stage s's table; twsize() is the total */                  \
        static constexpr int twoff(int stage)               \
        {                                                                       \
            int off = 0, ns = radices[0];                                       \
            for (int t = 1; t < stage; t++) {                                   \
                off += ns * radices[t];                                         \
                ns *= radices[t];                                               \
            }                                                                   \
            return off;                                                         \
        }                                                                       \
        static constexpr int twsize() { return twoff(nstages); } \
    };
JERK_FFT_PLAN(128, 4, 8, 4)
JERK_FFT_PLAN(192, 4, 16, 3)
JERK_FFT_PLAN(256, 8, 8, 4)
JERK_FFT_PLAN(384, 8, 16, 3)
JERK_FFT_PLAN(512, 8, 16, 4)
JERK_FFT_PLAN(768, 16, 16, 3)
JERK_FFT_PLAN(1024, 16, 16, 4)
JERK_FFT_PLAN(1280, 16, 16, 5)
JERK_FFT_PLAN(2048, 16, 16, 8)
JERK_FFT_PLAN(4096, 16, 16, 16)
JERK_FFT_PLAN(5120, 16, 16, 4, 5)
JERK_FFT_PLAN(7680, 16, 16, 2, 3, 5)
JERK_FFT_PLAN(8192, 16, 16, 16, 2)
JERK_FFT_PLAN(10240, 16, 16, 8, 5)
JERK_FFT_PLAN(15360, 16, 16, 4, 3, 5)
#undef JERK_FFT_PLAN

template <int SIGN>
__device__ __forceinline__ float2 twiddle(const float2 *tw, int m)
{
    float2 w = tw[m];
    return SIGN > 0 ? make_float2(w.x, -w.y) : w;
}

// Shared-buffer index: one float2 of padding after every 16 elements (one
// 128-byte row of banks).  Runs of 16 elements that start on a multiple of
// 16 -- every warp's half in every stage here -- stay within distinct banks,
// and the stride-16 writes of the first stage (element 16 t + r) land on
// bank pair (t + r) mod 16, so every stage's accesses are conflict-free.
__host__ __device__ __forceinline__ constexpr int pad(int i) { return i + (i >> 4); }
template <int N>
__host__ __device__ constexpr int fft_buf_len() { return N + N / 16; }
__host__ __device__ constexpr int fft_buf_len_rt(int n) { return n + n / 16; }

template <int X>
struct IsPow2 {
    static constexpr bool value = X > 0 && (X & (X - 1)) == 0;
};

// Padded address of element base + c, where base and the constant c have no
// set bits in common (base < 2^k <= lowest set bit of c, as for j + r * NB
// with j < NB, or idxD + r * Ns with j % Ns < Ns): no carry crosses bit 4, so
//   pad(base + c) = pad(base) + c + (c >> 4)
// with the last two terms a compile-time constant -- the access is a
// register plus an immediate offset.  (Measured against an XOR swizzle that
// needs one XOR per access: equal at fftlen 2048, 6 % faster at 1280.)
__device__ __forceinline__ int pad_add(int pbase, int c)
{
    return pbase + c + (c >> 4);
}

// One middle stage, in place in buf.  Every thread of the block must call it
// (it holds two barriers); only threads with act == true (tid < T) work.
// The twiddles and the butterfly run before the first barrier: only the
// writes must wait until every thread has read its inputs.
template <int N, int SIGN, int T, int Ns, int R>
__device__ __forceinline__ void fft_stage_inplace(float2 *buf, const float2 *tw, int tid, bool act)
{
    constexpr int NB = N / R;
    constexpr int PER = (NB + T - 1) / T;
    float2 v[PER][R];
    if (act) {
#pragma unroll
        for (int p = 0; p < PER; p++) {
            const int j = tid + p * T;
            if (NB % T == 0 || j < NB) {
                if constexpr (IsPow2<NB>::value && NB >= 16) {
                    const int pj = pad(j);
#pragma unroll
                    for (int r = 0; r < R; r++)
                        v[p][r] = buf[pad_add(pj, r * NB)];
                } else {
#pragma unroll
                    for (int r = 0; r < R; r++)
                        v[p][r] = buf[pad(j + r * NB)];
                }
                const int k = j % Ns;
                if (Ns > 1) {
#pragma unroll
                    for (int r = 1; r < R; r++)
                        v[p][r] = cmul(v[p][r], twiddle<SIGN>(tw, r * Ns + k));
                }
                Dft<R, SIGN>::run(v[p]);
            }
        }
    }
    __syncthreads();
    if (act) {
#pragma unroll
        for (int p = 0; p < PER; p++) {
            const int j = tid + p * T;
            if (NB % T == 0 || j < NB) {
                const int k = j % Ns;
                const int idxD = (j / Ns) * Ns * R + k;
                if constexpr (IsPow2<Ns>::value && IsPow2<R>::value) {
                    const int pd = pad(idxD);
#pragma unroll
                    for (int r = 0; r < R; r++)
                        buf[pad_add(pd, r * Ns)] = v[p][r];
                } else {
#pragma unroll
                    for (int r = 0; r < R; r++)
                        buf[pad(idxD + r * Ns)] = v[p][r];
                }
            }
        }
    }
    __syncthreads();
}

// One middle stage from src to dst (separate buffers): no barrier inside;
// the caller syncs before dst is read and before src is written again.
template <int N, int SIGN, int T, int Ns, int R>
__device__ __forceinline__ void fft_stage_oop(const float2 *src, float2 *dst, const float2 *tw,
                                              int tid)
{
    constexpr int NB = N / R;
    static_assert(NB % T == 0 && IsPow2<NB>::value && NB >= 16 && IsPow2<Ns>::value &&
                      IsPow2<R>::value, "power-of-two stage, whole butterflies per thread");
    constexpr int PER = NB / T;
#pragma unroll
    for (int p = 0; p < PER; p++) {
        const int j = tid + p * T;
        float2 v[R];
        const int pj = pad(j);
#pragma unroll
        for (int r = 0; r < R; r++)
            v[r] = src[pad_add(pj, r * NB)];
        const int k = j % Ns;
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; r++)
                v[r] = cmul(v[r], twiddle<SIGN>(tw, r * Ns + k));
        }
        Dft<R, SIGN>::run(v);
        const int pd = pad((j / Ns) * Ns * R + k);
#pragma unroll
        for (int r = 0; r < R; r++)
            dst[pad_add(pd, r * Ns)] = v[r];
    }
}

// Last stage: Ns * R == N, so the output index of (j, r) is j + r * Ns.
// No barrier inside; the caller must sync before buf is written again.
template <int N, int SIGN, int T, int Ns, int R, class Out>
__device__ __forceinline__ void fft_stage_last(const float2 *buf, const float2 *tw, int tid,
                                               bool act, Out &out)
{
    constexpr int NB = N / R;
    constexpr int PER = (NB + T - 1) / T;
    static_assert(Ns * R == N, "last stage");
    if (!act)
        return;
#pragma unroll
    for (int p = 0; p < PER; p++) {
        const int j = tid + p * T;
        if (NB % T == 0 || j < NB) {
            float2 v[R];
            if constexpr (IsPow2<NB>::value && NB >= 16) {
                const int pj = pad(j);
#pragma unroll
                for (int r = 0; r < R; r++)
                    v[r] = buf[pad_add(pj, r * NB)];
            } else {
#pragma unroll
                for (int r = 0; r < R; r++)
                    v[r] = buf[pad(j + r * NB)];
            }
#pragma unroll
            for (int r = 1; r < R; r++)
                v[r] = cmul(v[r], twiddle<SIGN>(tw, r * Ns + j));
            Dft<R, SIGN>::run(v);
#pragma unroll
            for (int r = 0; r < R; r++)
                out(j + r * Ns, v[r]);
        }
    }
}

// Stages I..end (I == nstages - 1 is the last one).
template <int N, int SIGN, int T, int I, int Ns, bool LAST = (I == FftPlan<N>::nstages - 1)>
struct FftTail;

template <int N, int SIGN, int T, int I, int Ns>
struct FftTail<N, SIGN, T, I, Ns, true> {
    template <class Out>
    __device__ __forceinline__ static void run(float2 *buf, const float2 *tw, int tid, bool act,
                                               Out &out)
    {
        constexpr int R = FftPlan<N>::radices[I];
        constexpr int OFF = FftPlan<N>::twoff(I);
        fft_stage_last<N, SIGN, T, Ns, R>(buf, tw + OFF, tid, act, out);
    }
};

template <int N, int SIGN, int T, int I, int Ns>
struct FftTail<N, SIGN, T, I, Ns, false> {
    template <class Out>
    __device__ __forceinline__ static void run(float2 *buf, const float2 *tw, int tid, bool act,
                                               Out &out)
    {
        constexpr int R = FftPlan<N>::radices[I];
        constexpr int OFF = FftPlan<N>::twoff(I);
        fft_stage_inplace<N, SIGN, T, Ns, R>(buf, tw + OFF, tid, act);
        FftTail<N, SIGN, T, I + 1, Ns * R>::run(buf, tw, tid, act, out);
    }
};

// Full transform by the whole block.  Threads with tid < T = N / R0 own
// first-stage butterfly j = tid, whose inputs are in(r) for the element
// index m = tid + r * (N / R0), r in [0, R0).  Every thread of the block
// must call it (barriers); threads with tid >= T do no work.  buf[N] is
// shared memory.  When it returns, outputs have been handed to out(m, y) by
// the threads that computed them; the caller must __syncthreads() before
// buf is written again.  buf holds fft_buf_len<N>() float2; tw holds the
// per-stage tables of FftPlan<N> (fft_stage_twiddles on the host).
//
// mid() is called by every thread right after the first-stage barrier, when
// no thread will call in() again (the caller may then refill in()'s source).
template <int N, int SIGN, class In, class Out, class Mid>
__device__ __forceinline__ void fft_block(float2 *buf, const float2 *tw, int tid, In &in,
                                          Out &out, Mid &&mid)
{
    using P = FftPlan<N>;
    constexpr int R0 = P::R0;
    constexpr int T = P::T;
    const bool act = tid < T;
    if (act) {
        float2 v[R0];
#pragma unroll
        for (int r = 0; r < R0; r++)
            v[r] = in(r);
        Dft<R0, SIGN>::run(v);
        if constexpr (IsPow2<R0>::value) {
            const int pd = pad(tid * R0);
#pragma unroll
            for (int r = 0; r < R0; r++)
                buf[pad_add(pd, r)] = v[r];
        } else {
#pragma unroll
            for (int r = 0; r < R0; r++)
                buf[pad(tid * R0 + r)] = v[r];
        }
    }
    __syncthreads();
    mid();
    FftTail<N, SIGN, T, 1, R0>::run(buf, tw, tid, act, out);
}

template <int N, int SIGN, class In, class Out>
__device__ __forceinline__ void fft_block(float2 *buf, const float2 *tw, int tid, In &in,
                                          Out &out)
{
    fft_block<N, SIGN>(buf, tw, tid, in, out, [] {});
}

// ---------------------------------------------------------------------------
// Two transforms at once in the two lanes of sm_100's packed FP32
// instructions (add / sub / mul / fma .f32x2).  A Cp holds one complex value
// of each transform: re = (re of lane 0, re of lane 1), im likewise.  Each
// packed operation rounds every lane as its scalar form does (round to
// nearest even), so the two transforms are computed exactly as two scalar
// runs of the same operation sequence would be, with half the instructions.
struct Cp {
    float2 re, im;
};

__device__ __forceinline__ float2 bc(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b)
{
    float2 d;
    asm("{\n\t.reg .b64 pa, pb, pd;\n\t"
        "mov.b64 pa, {%2, %3};\n\t"
        "mov.b64 pb, {%4, %5};\n\t"
        "sub.rn.f32x2 pd, pa, pb;\n\t"
        "mov.b64 {%0, %1}, pd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ Cp padd(Cp a, Cp b) { return {add2(a.re, b.re), add2(a.im, b.im)}; }
__device__ __forceinline__ Cp psub(Cp a, Cp b) { return {sub2(a.re, b.re), sub2(a.im, b.im)}; }
// a + i b and a - i b
__device__ __forceinline__ Cp padd_i(Cp a, Cp b) { return {sub2(a.re, b.im), add2(a.im, b.re)}; }
__device__ __forceinline__ Cp psub_i(Cp a, Cp b) { return {add2(a.re, b.im), sub2(a.im, b.re)}; }
// a (c + i s) for a constant or table root shared by both lanes:
// (re c - im s, im c + re s), each part one product and one fused add
__device__ __forceinline__ Cp pmul(Cp a, float c, float s)
{
    return {fma2(a.re, bc(c), mul2(a.im, bc(-s))), fma2(a.im, bc(c), mul2(a.re, bc(s)))};
}

// Inverse (exponent sign +1) DFTs of radix 4, 8 and 5 on lane pairs; the
// output order is that of Dft<R, +1>.
__device__ __forceinline__ void pdft4(Cp &v0, Cp &v1, Cp &v2, Cp &v3)
{
    const Cp a = padd(v0, v2), b = psub(v0, v2), c = padd(v1, v3), e = psub(v1, v3);
    v0 = padd(a, c);
    v2 = psub(a, c);
    v1 = padd_i(b, e);
    v3 = psub_i(b, e);
}

__device__ __forceinline__ void pdft8(Cp *v)
{
    pdft4(v[0], v[2], v[4], v[6]);
    pdft4(v[1], v[3], v[5], v[7]);
    // now v[0, 2, 4, 6] = E[0..3], v[1, 3, 5, 7] = O[0..3]
    const float h = 0.70710678118654752440f;
    const Cp e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    const Cp o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    // W8 = h (1 + i):   W8 O1 = h (t.re, t.im),  t = (o.re - o.im, o.im + o.re)
    // W8^3 = h (-1 + i): W8^3 O3 = h (-u.re, u.im), u = (o.re + o.im, o.re - o.im)
    const float2 tr = sub2(o1.re, o1.im), ti = add2(o1.im, o1.re);
    const float2 ur = add2(o3.re, o3.im), ui = sub2(o3.re, o3.im);
    v[0] = padd(e0, o0);
    v[4] = psub(e0, o0);
    v[1] = {fma2(bc(h), tr, e1.re), fma2(bc(h), ti, e1.im)};
    v[5] = {fma2(bc(-h), tr, e1.re), fma2(bc(-h), ti, e1.im)};
    v[2] = padd_i(e2, o2);
    v[6] = psub_i(e2, o2);
    v[3] = {fma2(bc(-h), ur, e3.re), fma2(bc(h), ui, e3.im)};
    v[7] = {fma2(bc(h), ur, e3.re), fma2(bc(-h), ui, e3.im)};
}

// Radix 5, as in Dft<5, +1>: with a1 = v1 + v4, b1 = v1 - v4, a2 = v2 + v3,
// b2 = v2 - v3 (c1, c2 = cos 2pi/5, cos 4pi/5; s1, s2 = sin 2pi/5, sin 4pi/5)
//   v0 = v0 + a1 + a2
//   v1, v4 = v0 + c1 a1 + c2 a2 +/- i (s1 b1 + s2 b2)
//   v2, v3 = v0 + c2 a1 + c1 a2 +/- i (s2 b1 - s1 b2)
__device__ __forceinline__ void pdft5(Cp *v)
{
    const float c1 = 0.30901699437494742410f;   // cos(2 pi/5)
    const float c2 = -0.80901699437494742410f;  // cos(4 pi/5)
    const float s1 = 0.95105651629515357212f;   // sin(2 pi/5)
    const float s2 = 0.58778525229247312917f;   // sin(4 pi/5)
    const Cp a1 = padd(v[1], v[4]), b1 = psub(v[1], v[4]);
    const Cp a2 = padd(v[2], v[3]), b2 = psub(v[2], v[3]);
    const Cp x0 = v[0];
    const Cp p1 = {fma2(bc(c2), a2.re, fma2(bc(c1), a1.re, x0.re)),
                   fma2(bc(c2), a2.im, fma2(bc(c1), a1.im, x0.im))};
    const Cp p2 = {fma2(bc(c1), a2.re, fma2(bc(c2), a1.re, x0.re)),
                   fma2(bc(c1), a2.im, fma2(bc(c2), a1.im, x0.im))};
    const Cp t1 = {fma2(bc(s2), b2.re, mul2(bc(s1), b1.re)), fma2(bc(s2), b2.im, mul2(bc(s1), b1.im))};
    const Cp t2 = {fma2(bc(-s1), b2.re, mul2(bc(s2), b1.re)),
                   fma2(bc(-s1), b2.im, mul2(bc(s2), b1.im))};
    v[0] = {add2(add2(x0.re, a1.re), a2.re), add2(add2(x0.im, a1.im), a2.im)};
    v[1] = padd_i(p1, t1);
    v[4] = psub_i(p1, t1);
    v[2] = padd_i(p2, t2);
    v[3] = psub_i(p2, t2);
}

// Host: the per-stage twiddle tables of FftPlan<N>, forward sign, computed
// in double and rounded to float.
template <int N>
inline void fft_stage_twiddles(float2 *out)
{
    using P = FftPlan<N>;
    int ns = P::radices[0];
    for (int s = 1; s < P::nstages; s++) {
        const int R = P::radices[s];
        float2 *t = out + P::twoff(s);
        for (int r = 0; r < R; r++)
            for (int k = 0; k < ns; k++) {
                const double a = -2.0 * 3.14159265358979323846264338327950288 * (double)(r * k) /
                                 (double)(ns * R);
                t[r * ns + k] = make_float2((float)cos(a), (float)sin(a));
            }
        ns *= R;
    }
}

}  // namespace jerk
