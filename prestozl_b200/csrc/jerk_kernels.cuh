// Device-side data structures shared by the jerk-search kernels and the host
// plan (jerk_plan.cpp).  Plain structs, no torch types.
#pragma once

#include <cuda.h>  // CUtensorMap

#include <cstdint>

namespace jerk {

constexpr int kMaxSubs = 32;      // numharm <= 32 -> 1 + 31 subharmonic planes
constexpr int kMaxStages = 6;

// One subharmonic (harmnum / numharm) as laid out on the device.
struct SubDev {
    int numharm, harmnum;
    double harm_fract;        // harmnum / numharm, computed on the host
    int numz, numw;           // kernel grid (numkern_zdim, numkern_wdim)
    int fftlen;
    int halfwidth;            // kern[0][0].kern_half_width (bins)
    int stride;               // plane row stride in floats (>= max numrs, multiple of 4)
    int zlo, wlo;             // lowest z / w of this subharmonic's volume
    float pownorm;            // (float)(1.0 / (fftlen * fftlen))
    int twoff;                // offset (float2) of this fftlen's twiddle table
    long long kern_off;       // offset (float2) of kernel [0][0] in the bank
    long long plane_off;      // offset (floats) of the b = 0 volume in the batch planes
    long long plane_size;     // floats per volume (numw * numz * stride)
    long long data_off;       // offset (float2) of the b = 0 prepared chunk
    int zinds_off;            // offset of zinds (u16, fundamental numz entries)
    int wind_off;             // offset of wind (int, fundamental numw entries)
};

// One (rstep, subharmonic): where its chunk starts and how many r it yields.
struct StepDev {
    long long rlo;            // floor(calc_required_r(hf, fullrlo))
    double fullrlo;           // fundamental r of the rstep's first bin
    int numrs;
    int pad;
};

struct SearchDev {
    // spectrum
    const float2 *spec;
    long long numbins;
    long long lobin;          // obs lobin: bin 0 of spec
    // geometry
    int nsubs;
    int nstages;
    int corr_uselen;
    int numz0, numw0;         // fundamental volume dims
    int norm_type;
    float nph;
    float powcut[kMaxStages];
    // tables
    const SubDev *subs;
    const StepDev *steps;     // [rstep][nsubs], whole spectrum
    const float2 *bank;
    const float2 *twiddles;
    const uint16_t *zinds;
    const int *wind;
    // per-batch work
    long long first_rstep;    // rstep index of b = 0
    int nb;                   // rsteps in this batch
    float2 *prepped;          // prepared chunks
    float *planes;            // ffdot volumes
    uint16_t *rinds;          // [b][s][corr_uselen]
    // hits
    unsigned long long *hit_keys;
    float *hit_pows;
    unsigned int *hit_count;
    long long max_hits;
    unsigned int *status;     // bit 0: a subharmonic r index fell outside its row
                              // (or its TMA box); bit 1: a bounded wait on a bulk
                              // or tensor copy gave up
};

// Tensor maps of the harmonic sum's TMA path: subharmonic s's batch volumes
// as a 4-D tensor (r, z, w, b) and the box one CTA loads per z tile:
// W[s] r cells (a multiple of 4, starting at the tile's first r index rounded
// down to 4) by Z[s] z rows, at boxoff[s] floats into the shared buffer.
struct HarmTma {
    CUtensorMap map[kMaxSubs];
    int W[kMaxSubs];
    int Z[kMaxSubs];
    int boxoff[kMaxSubs];
    int box_floats;           // shared floats of all boxes (offsets 128-byte aligned)
    int box_bytes;            // bytes the tensor copies of one tile deliver
};

// One response kernel of the bank (jerk_bank.cu).
struct BankRow {
    long long off;     // float2 offset of the row in the bank
    int z, w;          // this kernel's f-dot and f-dot-dot
    int fftlen;
    int numkern;       // 2 * numbetween * w_resp_halfwidth(z, w)
    int num_pts;       // w != 0: length of the cosine series
};

// The corr_kernel launch for one fftlen covers the rows (w, z) of every
// subharmonic with that fftlen, numbered consecutively.
struct RowGroup {
    int n;                       // subharmonics in this fftlen group
    int sub[kMaxSubs];
    int rowstart[kMaxSubs + 1];  // prefix sums of numw * numz
};

// One merged launch over the current batches of several plans (a "wave"):
// flat CTA index x belongs to plan i for cta0[i] <= x < cta0[i + 1], and
// that plan's part runs exactly the CTAs its own launch would run, with its
// own arguments, so every plan's results are bitwise those of its own
// launches.  ny[i]: corr -- rstep chunks per kernel row; harmsum -- r blocks
// per w row.  Passed by value as a __grid_constant__ parameter.
constexpr int kMaxGroupPlans = 12;
struct GroupLaunch {
    int n;
    int cta0[kMaxGroupPlans + 1];
    int ny[kMaxGroupPlans];
    SearchDev P[kMaxGroupPlans];
    RowGroup G[kMaxGroupPlans];
    const float2 *fold[kMaxGroupPlans];     // corr at fftlen 2048: folded kernel rows
    const float2 *fold_tw[kMaxGroupPlans];  // and their twiddle tables
};
static_assert(sizeof(GroupLaunch) <= 30000, "kernel parameter space");

// Records msg as the text jerk_last_error returns and passes code back.
int set_error(int code, const char *msg);
// w_resp_halfwidth(z, w, LOWACC) (src/responses.c:49-84).
int w_resp_halfwidth_lowacc(double z, double w);

// The reference's fast inverse square root (src/misc_utils.c:293-304): the
// published bit-level first guess and one Newton step in float, in the
// operation order the reference build evaluates it (y * (1.5 - (0.5 x)(y y)),
// its compiler's reassociation under -ffast-math), each step rounded on its
// own (no FMA).
__device__ __forceinline__ float invsqrtf_ref(float x)
{
    const float y = __int_as_float(0x5f3759df - (__float_as_int(x) >> 1));
    const float yy = __fmul_rn(y, y);
    const float hx = __fmul_rn(0.5f, x);
    return __fmul_rn(y, __fsub_rn(1.5f, __fmul_rn(hx, yy)));
}

}  // namespace jerk
