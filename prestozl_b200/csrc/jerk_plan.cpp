// Host side of libjerk: search geometry, the device plan, the batch loop,
// candidate assembly, and the C ABI of include/jerk.h.
//
// The plan owns every device buffer of one search configuration (kernel bank,
// twiddles, lookup tables, per-batch volumes, hit buffer) so that a search
// allocates nothing per rstep (the reference allocates and frees per call,
// src/accel_utils_cu.c:451-455, 591-611).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "jerk.h"
#include "jerk_kernels.cuh"

namespace jerk {
size_t prep_smem_bytes(int maxfft);
cudaError_t launch_prep(const SearchDev &P, int maxfft, cudaStream_t st);
cudaError_t launch_corr(const SearchDev &P, int fftlen, const RowGroup &G, int rows,
                        cudaStream_t st);
cudaError_t launch_harmsum(const SearchDev &P, const HarmTma &T, bool prefetch, cudaStream_t st);
cudaError_t launch_harmsum_tma(const SearchDev &P, const HarmTma &T, int zt, cudaStream_t st);
size_t harmsum_tma_smem_bytes(const HarmTma &T, int nsubs, int numz0);
bool fftlen_supported(int n);
cudaError_t launch_prep_group(GroupLaunch M, int maxfft, cudaStream_t st);
cudaError_t launch_corr_group(GroupLaunch M, int fftlen, cudaStream_t st);
cudaError_t launch_harmsum_group(GroupLaunch M, int nstages, cudaStream_t st);
cudaError_t launch_wait_probe(unsigned int *status, cudaStream_t st);
int corr_wave_ctas(int fftlen);
bool fold_length(int N);
int fold_twiddle_size(int N);
void fold_twiddle_table(int N, float2 *out);
cudaError_t launch_fold_rows(int N, const float2 *bank, const long long *src, float2 *out,
                             int nrows, cudaStream_t st);
cudaError_t launch_corr_fold(int N, const SearchDev &P, const RowGroup &G, int rows,
                             const float2 *F, const float2 *ftw, cudaStream_t st);
cudaError_t launch_corr_fold_group(int N, GroupLaunch M, cudaStream_t st);

// The FFT lengths whose correlation runs on folded kernel rows, and a
// length's slot in a plan's per-length fold arrays (-1: not folded).
constexpr int kFoldLens[2] = {2048, 1280};
static int fold_slot(int N)
{
    for (int i = 0; i < 2; i++)
        if (kFoldLens[i] == N)
            return i;
    return -1;
}
int harmsum_wave_ctas(int nstages);
int fft_twiddle_size(int N);
void fft_twiddle_table(int N, float2 *out);
cudaError_t launch_bank_response(const BankRow *rows, int nrows, int max_pts, float2 *bank,
                                 cudaStream_t st);
cudaError_t launch_bank_fft_any(int N, const BankRow *rows, int first, int count, const float2 *tw,
                                int twoff, float2 *bank, cudaStream_t st);
}  // namespace jerk

using namespace jerk;

// ---------------------------------------------------------------------------
// errors

static thread_local std::string g_err;

static int fail(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

static int cuda_fail(cudaError_t e, const char *what)
{
    return fail(JERK_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define JERK_CUDA(call)                                  \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess)                           \
            return cuda_fail(e_, #call);                 \
    } while (0)

extern "C" const char *jerk_last_error(void) { return g_err.c_str(); }

// Error reporting for the entry points compiled in other files.
int jerk::set_error(int code, const char *msg) { return fail(code, msg); }
extern "C" void jerk_free(void *p) { free(p); }

// ---------------------------------------------------------------------------
// Reference index arithmetic (src/accel_utils.c:36-97), host side.

static constexpr double kDR = 0.5;
static constexpr int kRDR = 2;
static constexpr int kDZ = 2;
static constexpr double kRDZ = 0.5;
static constexpr int kDW = 20;
static constexpr double kRDW = 0.05;
static constexpr double kDblCorrect = 1e-14;
static constexpr double kClosestR = 15.0;

static inline int nearest_int(double x) { return (int)(x < 0 ? x - 0.5 : x + 0.5); }
static inline double calc_required_r(double hf, double rfull) { return rint(kRDR * rfull * hf) * kDR; }
static inline int calc_required_z(double hf, double zfull) { return nearest_int(kRDZ * zfull * hf) * kDZ; }
static inline int calc_required_w(double hf, double wfull) { return nearest_int(kRDW * wfull * hf) * kDW; }
static inline int index_from_z(double z, double loz) { return (int)((z - loz) * kRDZ + kDblCorrect); }
static inline int index_from_w(double w, double low) { return (int)((w - low) * kRDW + kDblCorrect); }

// src/responses.c:27-84 (LOWACC)
static int z_resp_halfwidth(double z) { return (int)(0.5 * 1.1 * fabs(z)) + 16; }
static int w_resp_halfwidth(double z, double w)
{
    if (fabs(w) < 1.0e-7)
        return z_resp_halfwidth(z);
    const double r0 = 0.5 * (w / 6.0 - z), r1 = 0.5 * (w / 6.0 + z);
    double maxdev = fabs(r0) > fabs(r1) ? fabs(r0) : fabs(r1);
    const double u_ext = 0.5 - z / w;
    if (u_ext > 0.0 && u_ext < 1.0) {
        const double z0 = z - w / 2.0;
        const double r_ext = 0.5 * w * u_ext * u_ext + z0 * u_ext + r0;
        maxdev = fabs(r_ext) > maxdev ? fabs(r_ext) : maxdev;
    }
    return (int)(1.1 * maxdev) + 16;
}

int jerk::w_resp_halfwidth_lowacc(double z, double w) { return w_resp_halfwidth(z, w); }

static long long next2_to_n(long long x)
{
    long long n = 1;
    while (n < x)
        n <<= 1;
    return n;
}

// src/corr_prep.c:3-35
static int next_good_fftlen(int N)
{
    static const int lens[17] = {128, 192, 256, 384, 512, 768, 1024, 1280, 2048,
                                 4096, 5120, 7680, 10240, 12288, 15360, 16384, 25600};
    int ii = 0;
    if (N <= lens[0])
        return lens[0];
    if (N > lens[16])
        return (int)next2_to_n(N);
    while (N > lens[ii])
        ii++;
    return lens[ii];
}

static int fftlen_from_kernwidth(int kw)
{
    if (kw < 6) return 128;
    if (kw < 52) return 256;
    if (kw < 67) return 512;
    if (kw < 378) return 1024;
    if (kw < 664) return 2048;
    if (kw < 1672) return 4096;
    if (kw < 3015) return 10240;
    if (kw < 3554) return 15360;
    if (kw < 6000) return 25600;
    return (int)next2_to_n(kw * 5);
}

// ---------------------------------------------------------------------------
// Statistics: candidate_sigma / power_for_sigma (src/characteristics.c:400-705)
// for the integer numsum the search uses, written from the published
// formulas the reference's code evaluates.

// ln Gamma(a, z), the upper incomplete gamma function, for large z by its
// asymptotic series (Abramowitz & Stegun 6.5.32):
//   Gamma(a, z) ~ z^(a-1) e^(-z) sum_k (a-1)(a-2)...(a-k) / z^k,
// summed until a term drops below 1e-15.
static double log_upper_gamma_large_z(double a, double z)
{
    double sum = 1.0, coef = 1.0, term = 1.0;
    for (int k = 1; fabs(term) > 1e-15; k++) {
        coef *= (a - k);
        term = coef / pow(z, k);
        sum += term;
    }
    return (a - 1.0) * log(z) - z + log(sum);
}

// ln Gamma(z) by Stirling's series (Abramowitz & Stegun 6.1.41), to the
// z^-7 term: (z - 1/2) ln z - z + ln(2 pi)/2 + 1/(12 z) - 1/(360 z^3)
// + 1/(1260 z^5) - 1/(1680 z^7).
static double log_gamma_stirling(double z)
{
    const double half_log_2pi = 0.91893853320467274178;
    const double u = 1.0 / (z * z);
    const double series =
        (((-1.0 / 1680.0) * u + 1.0 / 1260.0) * u - 1.0 / 360.0) * u + 1.0 / 12.0;
    return (z - 0.5) * log(z) - z + half_log_2pi + series / z;
}

// Q(a, x) for integer a: exp(-x) sum_{n<a} x^n / n!
static double q_gamma_int(int a, double x)
{
    if (x <= 0.0)
        return 1.0;
    double t = exp(-x), sum = t;
    for (int n = 1; n < a; n++) {
        t = t * x / n;
        sum += t;
    }
    return sum;
}

static double chi2_logp(double chi2, double dof)
{
    if (chi2 <= 0.0)
        return -INFINITY;
    if (chi2 / dof > 15.0 || (dof > 150 && chi2 / dof > 6.0))
        return log_upper_gamma_large_z(0.5 * dof, 0.5 * chi2) -
               log_gamma_stirling(0.5 * dof);
    return log(q_gamma_int((int)(0.5 * dof + 0.5), 0.5 * chi2));
}

// x with 1 - Phi(x) = q, full double precision
static double upper_normal_quantile(double q)
{
    double lo = -40.0, hi = 40.0, x = 0.0;
    for (int it = 0; it < 200; it++) {
        x = 0.5 * (lo + hi);
        if (0.5 * erfc(x / M_SQRT2) > q)
            lo = x;
        else
            hi = x;
        if (hi - lo < 1e-15 * (fabs(x) + 1.0))
            break;
    }
    for (int it = 0; it < 3; it++) {
        const double dens = exp(-0.5 * x * x) / sqrt(2.0 * M_PI);
        if (dens <= 0.0)
            break;
        x += (0.5 * erfc(x / M_SQRT2) - q) / dens;
    }
    return x;
}

static double equivalent_gaussian_sigma(double logp)
{
    double x;
    if (logp < -600.0) {
        // the rational approximation of the normal quantile, Abramowitz &
        // Stegun 26.2.23, on log p (|error| < 4.5e-4)
        const double t = sqrt(-2.0 * logp);
        const double num = 2.515517 + t * (0.802853 + t * 0.010328);
        const double den = 1.0 + t * (1.432788 + t * (0.189269 + t * 0.001308));
        x = t - num / den;
    } else {
        const double q = exp(logp);
        /* p = 1 - q < 0 has no normal quantile: the reference's cdfnor2 gives
           NaN there, and -inf (clamped to 0) at q == 1 */
        if (q > 1.0)
            return NAN;
        if (q == 1.0)
            return 0.0;
        x = upper_normal_quantile(q);
    }
    return x < 0.0 ? 0.0 : x;
}

extern "C" double jerk_candidate_sigma(double power, int numsum, double numtrials)
{
    if (power <= 0.0)
        return 0.0;
    double logp = chi2_logp(2.0 * power, 2.0 * numsum);
    logp += log(numtrials);
    return equivalent_gaussian_sigma(logp);
}

extern "C" double jerk_power_for_sigma(double sigma, int numsum, double numtrials)
{
    const double q = 0.5 * erfc(sigma / M_SQRT2) / numtrials;
    const double logq = log(q);
    double lo = 0.0, hi = 1.0;
    while (log(q_gamma_int(numsum, hi)) > logq)
        hi *= 2.0;
    for (int it = 0; it < 200; it++) {
        const double mid = 0.5 * (lo + hi);
        if (log(q_gamma_int(numsum, mid)) > logq)
            lo = mid;
        else
            hi = mid;
        if (hi - lo <= 1e-15 * hi)
            break;
    }
    return 0.5 * (lo + hi);
}

// ---------------------------------------------------------------------------
// Geometry (the sizing part of create_accelobs, src/accel_utils.c:1795-2004)

extern "C" int jerk_obs_from_params(long long numbins, long long N, double dt, int zmax, int wmax,
                                    int wmax_given, int numharm, float sigma, double flo,
                                    double fhi, jerk_obs *obs, int *fftlen_out,
                                    int *maxkernlen_out)
{
    if (!obs || numbins < 2 || dt <= 0.0)
        return fail(JERK_EINVAL, "jerk_obs_from_params: bad arguments");
    if (numharm != 1 && numharm != 2 && numharm != 4 && numharm != 8 && numharm != 16 &&
        numharm != 32)
        return fail(JERK_EINVAL, "numharm must be a power of two <= 32");
    memset(obs, 0, sizeof(*obs));
    if (zmax % kDZ)
        zmax = (zmax / kDZ + 1) * kDZ;
    const double T = dt * (double)N;
    obs->numbins = numbins;
    obs->lobin = 0;
    int stages = 0;
    while ((1 << stages) < numharm)
        stages++;
    obs->numharmstages = stages + 1;
    obs->numz = (zmax / kDZ) * 2 + 1;
    double whi = 0.0;
    int numw = 0;
    if (wmax_given) {
        if (wmax % kDW)
            wmax = (wmax / kDW + 1) * kDW;
        whi = wmax;
        numw = (wmax / kDW) * 2 + 1;
        if (wmax == 0)
            numw = 0;
    } else {
        wmax = 0;
    }
    obs->numw = numw;
    obs->zlo = -zmax;
    obs->wlo = -whi;
    obs->rlo = floor(flo * T);
    if (obs->rlo < obs->lobin)
        obs->rlo = obs->lobin;
    if (obs->rlo > numbins - 1)
        return fail(JERK_EINVAL, "flo is above the highest frequency");
    obs->highestbin = numbins - 1;
    obs->highestbin = (long long)ceil(fhi * T);
    if (obs->highestbin > numbins - 1)
        obs->highestbin = numbins - 1;
    const double rhi = (double)obs->highestbin;
    if (obs->highestbin < obs->rlo)
        return fail(JERK_EINVAL, "fhi is below flo");
    const double dz = kDZ, dw = wmax_given ? kDW : 0.0;
    for (int ii = 0; ii < obs->numharmstages; ii++) {
        const int h = 1 << ii;
        if (obs->numz == 1 && obs->numw == 0)
            obs->numindep[ii] = (long long)((rhi - obs->rlo) / h);
        else if (obs->numz > 1 && obs->numw == 0)
            obs->numindep[ii] = (long long)((rhi - obs->rlo) * (obs->numz + 1) * (dz / 6.95) / h);
        else
            obs->numindep[ii] = (long long)((rhi - obs->rlo) * (obs->numz + 1) * (dz / 6.95) *
                                            (obs->numw + 1) * (dw / 44.2) / h);
        obs->powcut[ii] = (float)jerk_power_for_sigma(sigma, h, (double)obs->numindep[ii]);
    }
    const int maxkernlen = 2 * 2 * w_resp_halfwidth(zmax, whi);
    int fftlen = fftlen_from_kernwidth(maxkernlen);
    if (fftlen < 2048)
        fftlen = 2048;
    int uselen = fftlen - maxkernlen;
    if (uselen % kRDR)
        uselen = uselen / kRDR * kRDR;
    obs->corr_uselen = uselen;
    if (fftlen_out)
        *fftlen_out = fftlen;
    if (maxkernlen_out)
        *maxkernlen_out = maxkernlen;
    return JERK_OK;
}

extern "C" int jerk_subharm_count(int numharmstages)
{
    return numharmstages < 1 ? 0 : (1 << (numharmstages - 1));
}

// Bank order (src/accel_utils.c:236-282): (1/1), (1/2), (1/4), (3/4), (1/8), ...
static void index_to_harm(int index, int *numharm, int *harmnum)
{
    if (index == 0) {
        *numharm = 1;
        *harmnum = 1;
        return;
    }
    int stage = 1;
    while (index >= (1 << stage))
        stage++;
    // stage s holds subharmonics 2^(s-1) .. 2^s - 1, harm = 2*(index - 2^(s-1)) + 1
    *numharm = 1 << stage;
    *harmnum = 2 * (index - (1 << (stage - 1))) + 1;
}

extern "C" int jerk_subharm_sizes(const jerk_obs *obs, int fftlen, int index, jerk_subharm *out)
{
    if (!obs || !out || index < 0 || index >= jerk_subharm_count(obs->numharmstages))
        return fail(JERK_EINVAL, "jerk_subharm_sizes: bad index");
    int nh, hn;
    index_to_harm(index, &nh, &hn);
    const double hf = (double)hn / (double)nh;
    const int zmax = (int)-obs->zlo, wmax = (int)-obs->wlo;
    memset(out, 0, sizeof(*out));
    out->numharm = nh;
    out->harmnum = hn;
    out->zmax = calc_required_z(hf, zmax);
    out->wmax = calc_required_w(hf, wmax);
    out->numz = (out->zmax / kDZ) * 2 + 1;
    out->numw = (out->wmax / kDW) * 2 + 1;
    if (nh == 1 && hn == 1) {
        out->fftlen = fftlen;
    } else {
        const int bins_needed = (int)ceil(obs->corr_uselen * hf) + 2;
        const int end_effects = 2 * 2 * w_resp_halfwidth(calc_required_z(hf, zmax),
                                                         calc_required_w(hf, wmax));
        out->fftlen = next_good_fftlen(bins_needed + end_effects);
    }
    out->halfwidth = w_resp_halfwidth((double)-out->zmax, (double)-out->wmax);
    out->kernels = nullptr;
    return JERK_OK;
}

// ---------------------------------------------------------------------------
// Candidate list: insert_new_accelcand (src/accel_utils.c:382-480).
//
// The reference walks a linked list from its head to the first node with
// r >= rr (or to the last node).  The list is not always sorted -- when the
// walk ends at the last node and only the node before it is overwritten, a
// larger r lands before a smaller one -- so the walk cannot be replaced by a
// binary search.  CandList keeps the list in blocks with each block's max r:
// "first node with r >= rr" skips whole blocks whose max is below rr, which
// gives the walk's exact answer in O(sqrt n) instead of O(n).

namespace {

class CandList {
  public:
    struct Pos {
        size_t b, o;
    };

    bool empty() const { return n_ == 0; }

    // the reference walk's stopping node
    Pos walk(double rr) const
    {
        for (size_t b = 0; b < blocks_.size(); b++) {
            if (blocks_[b].maxr >= rr) {
                const auto &v = blocks_[b].v;
                for (size_t o = 0; o < v.size(); o++)
                    if (!(v[o].r < rr))
                        return {b, o};
            }
        }
        return last();
    }
    Pos last() const { return {blocks_.size() - 1, blocks_.back().v.size() - 1}; }
    bool is_last(Pos p) const { return p.b == blocks_.size() - 1 && p.o == blocks_[p.b].v.size() - 1; }
    bool has_prev(Pos p) const { return p.o > 0 || p.b > 0; }
    Pos prev(Pos p) const { return p.o > 0 ? Pos{p.b, p.o - 1} : Pos{p.b - 1, blocks_[p.b - 1].v.size() - 1}; }
    const jerk_cand &at(Pos p) const { return blocks_[p.b].v[p.o]; }

    void push_back(const jerk_cand &c)
    {
        if (blocks_.empty() || blocks_.back().v.size() >= 2 * kBlock)
            blocks_.push_back(Block{});
        Block &B = blocks_.back();
        B.v.push_back(c);
        B.maxr = B.v.size() == 1 ? c.r : std::max(B.maxr, c.r);
        n_++;
    }
    void replace(Pos p, const jerk_cand &c)
    {
        Block &B = blocks_[p.b];
        B.v[p.o] = c;
        remax(B);
    }
    void insert_before(Pos p, const jerk_cand &c)
    {
        Block &B = blocks_[p.b];
        B.v.insert(B.v.begin() + p.o, c);
        B.maxr = std::max(B.maxr, c.r);
        n_++;
        if (B.v.size() > 2 * kBlock)
            split(p.b);
    }
    void erase(Pos p)
    {
        Block &B = blocks_[p.b];
        B.v.erase(B.v.begin() + p.o);
        n_--;
        if (B.v.empty())
            blocks_.erase(blocks_.begin() + p.b);
        else
            remax(B);
    }
    void export_to(std::vector<jerk_cand> &out) const
    {
        out.clear();
        out.reserve(n_);
        for (const auto &B : blocks_)
            out.insert(out.end(), B.v.begin(), B.v.end());
    }

  private:
    static constexpr size_t kBlock = 256;
    struct Block {
        std::vector<jerk_cand> v;
        double maxr = -INFINITY;
    };
    static void remax(Block &B)
    {
        double m = -INFINITY;
        for (const auto &c : B.v)
            m = std::max(m, c.r);
        B.maxr = m;
    }
    void split(size_t b)
    {
        Block nb;
        Block &B = blocks_[b];
        nb.v.assign(B.v.begin() + kBlock, B.v.end());
        B.v.resize(kBlock);
        remax(B);
        remax(nb);
        blocks_.insert(blocks_.begin() + b + 1, std::move(nb));
    }
    std::vector<Block> blocks_;
    size_t n_ = 0;
};

bool insert_cand(CandList &L, const jerk_cand &v)
{
    if (L.empty()) {
        L.push_back(v);
        return true;
    }
    const CandList::Pos tmp = L.walk(v.r);
    const bool have_prev = L.has_prev(tmp);
    const double next_diff = fabs(v.r - L.at(tmp).r);
    const double prev_diff = have_prev ? fabs(v.r - L.at(L.prev(tmp)).r) : kClosestR + 1.0;
    bool added = false;
    if (prev_diff < kClosestR) {
        const CandList::Pos prev = L.prev(tmp);
        if (L.at(prev).sigma < v.sigma) {
            L.replace(prev, v);
            added = true;
        }
        if (next_diff < kClosestR && L.at(tmp).sigma < v.sigma) {
            if (added)
                L.erase(tmp);
            else {
                L.replace(tmp, v);
                added = true;
            }
        }
    } else if (next_diff < kClosestR) {
        if (L.at(tmp).sigma < v.sigma) {
            L.replace(tmp, v);
            added = true;
        }
    } else {
        added = true;
        if (L.is_last(tmp) && L.at(tmp).r < v.r - kClosestR)
            L.push_back(v);
        else
            L.insert_before(tmp, v);
    }
    return added;
}

long long export_list(const CandList &CL, jerk_cand **out)
{
    std::vector<jerk_cand> L;
    CL.export_to(L);
    if (!out)
        return (long long)L.size();
    *out = (jerk_cand *)malloc(sizeof(jerk_cand) * (L.size() ? L.size() : 1));
    if (!*out)
        return -1;
    if (!L.empty())
        memcpy(*out, L.data(), sizeof(jerk_cand) * L.size());
    return (long long)L.size();
}

}  // namespace

extern "C" long long jerk_insert_hits(const jerk_cand *hits, long long nhits, jerk_cand **cands)
{
    CandList L;
    for (long long i = 0; i < nhits; i++)
        insert_cand(L, hits[i]);
    return export_list(L, cands);
}

// ---------------------------------------------------------------------------
// the per-stage twiddle tables of fftlen N's FFT plan (jerk_fft.cuh)

static void append_twiddles(int N, std::vector<float2> &tw)
{
    const size_t at = tw.size();
    tw.resize(at + fft_twiddle_size(N));
    fft_twiddle_table(N, tw.data() + at);
}

// ---------------------------------------------------------------------------
// Kernel bank (create_subharminfos / init_kernel, src/accel_utils.c:151-282)

extern "C" long long jerk_bank_elements(const jerk_subharm *subs, int nsubs)
{
    long long n = 0;
    for (int s = 0; s < nsubs; s++)
        n += (long long)subs[s].numw * subs[s].numz * subs[s].fftlen;
    return n;
}

extern "C" int jerk_device_alloc(long long bytes, void **out)
{
    if (!out || bytes <= 0)
        return fail(JERK_EINVAL, "jerk_device_alloc: bad argument");
    JERK_CUDA(cudaMalloc(out, (size_t)bytes));
    return JERK_OK;
}

extern "C" void jerk_device_free(void *p) { cudaFree(p); }

extern "C" int jerk_copy_to_host(void *dst, const void *src, long long bytes)
{
    JERK_CUDA(cudaMemcpy(dst, src, (size_t)bytes, cudaMemcpyDeviceToHost));
    return JERK_OK;
}

extern "C" int jerk_bank_generate(const jerk_subharm *subs, int nsubs, void *device_bank,
                                  void *stream)
{
    if (!subs || nsubs <= 0 || !device_bank)
        return fail(JERK_EINVAL, "jerk_bank_generate: bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    // rows grouped by fftlen so each FFT launch covers a contiguous range
    std::map<int, std::vector<BankRow>> byN;
    long long off = 0;
    int max_pts = 1;
    for (int s = 0; s < nsubs; s++) {
        const jerk_subharm &sh = subs[s];
        if (!fftlen_supported(sh.fftlen))
            return fail(JERK_EUNSUPPORTED, "unsupported fftlen " + std::to_string(sh.fftlen));
        for (int ii = 0; ii < sh.numw; ii++)
            for (int jj = 0; jj < sh.numz; jj++) {
                BankRow r{};
                r.z = -sh.zmax + jj * kDZ;
                r.w = -sh.wmax + ii * kDW;
                r.fftlen = sh.fftlen;
                const int hw = w_resp_halfwidth((double)r.z, (double)r.w);
                r.numkern = 2 * 2 * hw;
                r.num_pts = 0;
                if (fabs((double)r.w) >= 1e-4) {
                    r.num_pts = (int)next2_to_n(6 * hw + 200 + r.numkern / 2);
                    max_pts = std::max(max_pts, r.num_pts);
                }
                if (r.numkern > sh.fftlen)
                    return fail(JERK_EINVAL, "response wider than its fftlen");
                r.off = off + ((long long)ii * sh.numz + jj) * sh.fftlen;
                byN[sh.fftlen].push_back(r);
            }
        off += (long long)sh.numw * sh.numz * sh.fftlen;
    }
    if ((size_t)max_pts * sizeof(float) > 200 * 1024)
        return fail(JERK_EUNSUPPORTED, "response series too long for shared memory");
    std::vector<BankRow> rows;
    std::vector<std::pair<int, std::pair<int, int>>> groups;  // N, (first, count)
    std::vector<float2> tw;
    std::map<int, int> twoff;
    for (auto &kv : byN) {
        groups.push_back({kv.first, {(int)rows.size(), (int)kv.second.size()}});
        rows.insert(rows.end(), kv.second.begin(), kv.second.end());
        twoff[kv.first] = (int)tw.size();
        append_twiddles(kv.first, tw);
    }
    BankRow *d_rows = nullptr;
    float2 *d_tw = nullptr;
    int rc = JERK_OK;
    cudaError_t e = cudaMalloc(&d_rows, sizeof(BankRow) * rows.size());
    if (e == cudaSuccess)
        e = cudaMalloc(&d_tw, sizeof(float2) * tw.size());
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_rows, rows.data(), sizeof(BankRow) * rows.size(),
                            cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_tw, tw.data(), sizeof(float2) * tw.size(), cudaMemcpyHostToDevice,
                            st);
    if (e == cudaSuccess)
        e = launch_bank_response(d_rows, (int)rows.size(), max_pts, (float2 *)device_bank, st);
    for (size_t g = 0; g < groups.size() && e == cudaSuccess; g++)
        e = launch_bank_fft_any(groups[g].first, d_rows, groups[g].second.first,
                                groups[g].second.second, d_tw, twoff[groups[g].first],
                                (float2 *)device_bank, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        rc = cuda_fail(e, "jerk_bank_generate");
    cudaFree(d_rows);
    cudaFree(d_tw);
    return rc;
}

// ---------------------------------------------------------------------------
// The plan

// per kernel class: launches, device time (CUDA events on the plan's stream,
// only while profiling is on), and algorithmic bytes / flops of the launches
struct KernelClass {
    std::string name;
    long long launches = 0;
    double ms = 0.0, bytes = 0.0, flops = 0.0;
};

struct PendingTiming {
    int cls;
    cudaEvent_t start, stop;
};

struct jerk_plan {
    int device = 0;
    cudaStream_t stream = nullptr;   // prep + correlation (and the caller's work)
    bool own_stream = false;
    jerk_obs obs{};
    int nsubs = 0, maxfft = 0, batch = 8;
    // harmonic-sum kernel (jerk_config.harm_mode, resolved): 1 gather,
    // 2 gather + TMA L2 prefetch, 3 / 4 TMA tiles of harm_tile (8 / 16) rows;
    // tma holds the tensor maps of modes 2-4
    int harm_mode = 1;
    int harm_tile = 16;
    std::unique_ptr<HarmTma> tma;
    // graph mode: a whole pass captured once per (first, count) and replayed;
    // the spectrum is always staged into d_spec so one graph fits any input
    bool use_graph = false;
    cudaGraphExec_t graph_exec = nullptr;
    long long graph_first = -1, graph_count = -1;
    long long graph_replays = 0;
    int zlo0 = 0, wlo0 = 0;
    long long nrsteps = 0;
    std::vector<jerk_subharm> subs;
    std::vector<SubDev> hsubs;
    std::vector<StepDev> hsteps;  // [nrsteps][nsubs]
    std::map<int, std::vector<int>> groups;  // fftlen -> subs
    // device
    float2 *d_bank = nullptr;
    bool own_bank = false;
    float2 *d_tw = nullptr;
    // per folded length (kFoldLens): the rows folded for the half-length
    // correlation, and the offset of its twiddle tables in d_tw
    float2 *d_fold[2] = {nullptr, nullptr};
    long long fold_floats2[2] = {0, 0};
    int fold_twoff[2] = {-1, -1};
    SubDev *d_subs = nullptr;
    StepDev *d_steps = nullptr;
    uint16_t *d_zinds = nullptr;
    int *d_wind = nullptr;
    float2 *d_prepped = nullptr;
    float *d_planes = nullptr;
    uint16_t *d_rinds = nullptr;
    float2 *d_spec = nullptr;
    long long spec_cap = 0;
    unsigned long long *d_hit_keys = nullptr;
    float *d_hit_pows = nullptr;
    unsigned int *d_hit_count = nullptr;
    unsigned int *d_status = nullptr;
    int wait_probe = 0;                // jerk_debug_wait_probe
    long long max_hits = 0;
    long long plane_floats = 0, prepped_f2 = 0;
    // a search pass being enqueued batch by batch
    struct Pass {
        SearchDev a{};
        long long first = 0, count = 0, next = 0, nbatch = 0, ndone = 0;
        bool all_enqueued = false;
        bool capturing = false;  // being recorded into a graph: no host-side event queries
        int error = 0;  // first enqueue failure (the pass is then abandoned)
    } pass;
    static constexpr int kRing = 16;
    cudaEvent_t ev_batch[kRing] = {};  // harmonic sum of batch n done (n % kRing)
    // asynchronous search in flight (jerk_search_async / jerk_search_collect)
    bool in_flight = false;
    const float2 *inflight_spec = nullptr;
    long long inflight_first = 0, inflight_count = 0;
    unsigned int *h_counts = nullptr;  // pinned: hit count, status
    cudaEvent_t ev_done = nullptr;
    // instrumentation
    bool profiling = false;
    std::vector<KernelClass> classes;
    std::map<std::string, int> class_index;
    std::vector<PendingTiming> pending;
    std::vector<cudaEvent_t> event_pool;
    long long h2d_bytes = 0, d2h_bytes = 0;
};

static int kclass(jerk_plan *p, const std::string &name)
{
    auto it = p->class_index.find(name);
    if (it != p->class_index.end())
        return it->second;
    KernelClass k;
    k.name = name;
    p->classes.push_back(k);
    p->class_index[name] = (int)p->classes.size() - 1;
    return (int)p->classes.size() - 1;
}

static cudaEvent_t take_event(jerk_plan *p)
{
    if (!p->event_pool.empty()) {
        cudaEvent_t e = p->event_pool.back();
        p->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Bracket one launch: returns a token to pass to launch_end.
static int launch_begin(jerk_plan *p, int cls, double bytes, double flops)
{
    KernelClass &k = p->classes[cls];
    k.launches++;
    k.bytes += bytes;
    k.flops += flops;
    if (!p->profiling)
        return -1;
    PendingTiming t{cls, take_event(p), take_event(p)};
    cudaEventRecord(t.start, p->stream);
    p->pending.push_back(t);
    return (int)p->pending.size() - 1;
}

static void launch_end(jerk_plan *p, int token)
{
    if (token >= 0)
        cudaEventRecord(p->pending[token].stop, p->stream);
}

// after a stream synchronisation: fold the recorded intervals into the classes
static void collect_timings(jerk_plan *p)
{
    for (auto &t : p->pending) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, t.start, t.stop) == cudaSuccess)
            p->classes[t.cls].ms += ms;
        p->event_pool.push_back(t.start);
        p->event_pool.push_back(t.stop);
    }
    p->pending.clear();
}

extern "C" int jerk_plan_set_profiling(jerk_plan *p, int on)
{
    if (!p)
        return fail(JERK_EINVAL, "null plan");
    p->profiling = on != 0;
    return JERK_OK;
}

extern "C" void jerk_plan_reset_stats(jerk_plan *p)
{
    if (!p)
        return;
    for (auto &k : p->classes) {
        k.launches = 0;
        k.ms = k.bytes = k.flops = 0.0;
    }
    p->h2d_bytes = p->d2h_bytes = 0;
}

extern "C" int jerk_plan_kernel_stats(const jerk_plan *p, int max, jerk_kernel_stat *out)
{
    if (!p)
        return 0;
    int n = 0;
    for (const auto &k : p->classes) {
        if (n < max && out) {
            memset(&out[n], 0, sizeof(out[n]));
            strncpy(out[n].name, k.name.c_str(), sizeof(out[n].name) - 1);
            out[n].launches = k.launches;
            out[n].ms = k.ms;
            out[n].bytes = k.bytes;
            out[n].flops = k.flops;
        }
        n++;
    }
    return n;
}

extern "C" void jerk_plan_transfer_stats(const jerk_plan *p, long long *h2d, long long *d2h)
{
    if (h2d)
        *h2d = p ? p->h2d_bytes : 0;
    if (d2h)
        *d2h = p ? p->d2h_bytes : 0;
}

static void drop_graph(jerk_plan *p)
{
    if (p->graph_exec)
        cudaGraphExecDestroy(p->graph_exec);
    p->graph_exec = nullptr;
    p->graph_first = p->graph_count = -1;
}

static void plan_free_device(jerk_plan *p)
{
    if (p->own_bank)
        cudaFree(p->d_bank);
    cudaFree(p->d_tw);
    cudaFree(p->d_fold[0]);
    cudaFree(p->d_fold[1]);
    cudaFree(p->d_subs);
    cudaFree(p->d_steps);
    cudaFree(p->d_zinds);
    cudaFree(p->d_wind);
    cudaFree(p->d_prepped);
    cudaFree(p->d_planes);
    cudaFree(p->d_rinds);
    cudaFree(p->d_spec);
    cudaFree(p->d_hit_keys);
    cudaFree(p->d_hit_pows);
    cudaFree(p->d_hit_count);
    cudaFree(p->d_status);
}

extern "C" void jerk_plan_destroy(jerk_plan *p)
{
    if (!p)
        return;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(p->device);
    if (p->stream)
        cudaStreamSynchronize(p->stream);
    drop_graph(p);
    plan_free_device(p);
    for (auto &t : p->pending) {
        cudaEventDestroy(t.start);
        cudaEventDestroy(t.stop);
    }
    for (auto e : p->event_pool)
        cudaEventDestroy(e);
    if (p->ev_done)
        cudaEventDestroy(p->ev_done);
    for (int i = 0; i < jerk_plan::kRing; i++)
        if (p->ev_batch[i])
            cudaEventDestroy(p->ev_batch[i]);
    if (p->h_counts)
        cudaFreeHost(p->h_counts);
    if (p->own_stream && p->stream)
        cudaStreamDestroy(p->stream);
    cudaSetDevice(cur);
    delete p;
}

static int alloc_hits(jerk_plan *p, long long cap)
{
    drop_graph(p);  // the captured pass holds the old hit buffers
    cudaFree(p->d_hit_keys);
    cudaFree(p->d_hit_pows);
    p->d_hit_keys = nullptr;
    p->d_hit_pows = nullptr;
    JERK_CUDA(cudaMalloc(&p->d_hit_keys, sizeof(unsigned long long) * cap));
    JERK_CUDA(cudaMalloc(&p->d_hit_pows, sizeof(float) * cap));
    p->max_hits = cap;
    return JERK_OK;
}

static long long count_rsteps(const jerk_obs &o)
{
    const int rstep = (int)(o.corr_uselen * kDR);
    long long n = 0;
    double startr = o.rlo;
    while (startr + rstep < (double)o.highestbin) {
        n++;
        startr += rstep;
    }
    return n;
}

extern "C" long long jerk_num_rsteps(const jerk_plan *p) { return p ? p->nrsteps : 0; }

// cuTensorMapEncodeTiled from the driver, without linking libcuda.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)f;
    });
    return fn;
}

// The harmonic sum's TMA boxes and tensor maps (HarmTma in jerk_kernels.cuh).
// A tile covers kThreads fundamental r (one CTA) x harm_tile fundamental z.
// Subharmonic index steps are 0 or 1 per fundamental step (harm_fract <= 1),
// so over n steps an index grows by at most floor(n * harm_fract) + 1: the box
// spans that + 1 cells / rows, plus 3 cells for rounding its first r index
// down to a multiple of 4.  For the tile kernel (in_smem) the boxes must fit
// next to the z tables in shared memory; if they do not, or the driver has no
// tensor-map encoder, tma stays null and the plan uses the gather kernel.
static int build_harm_tma(jerk_plan *p, bool in_smem)
{
    constexpr int kThreads = 128;  // harmonic-sum CTA width (kHarmThreads)
    auto T = std::make_unique<HarmTma>();
    memset(T.get(), 0, sizeof(HarmTma));
    const int zt = p->harm_tile;
    int off = 0;
    long long bytes = 0;
    for (int s = 0; s < p->nsubs; s++) {
        const SubDev &d = p->hsubs[s];
        const double hf = d.harm_fract;
        const int W = s == 0 ? kThreads : ((int)floor((kThreads - 1) * hf) + 5 + 3) & ~3;
        const int Z = s == 0 ? zt : (int)floor((zt - 1) * hf) + 2;
        if (W > 256 || Z > 256)
            return JERK_OK;
        T->W[s] = W;
        T->Z[s] = Z;
        T->boxoff[s] = off;
        off += (W * Z + 31) & ~31;  // 128-byte aligned boxes
        bytes += 4LL * W * Z;
    }
    T->box_floats = off;
    T->box_bytes = (int)bytes;
    const size_t smem = harmsum_tma_smem_bytes(*T, p->nsubs, p->subs[0].numz);
    if (in_smem && smem + 1024 > 200 * 1024)
        return JERK_OK;  // boxes too large: gather kernel
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc)
        return JERK_OK;  // no driver entry point: gather kernel
    for (int s = 0; s < p->nsubs; s++) {
        const SubDev &d = p->hsubs[s];
        const cuuint64_t dims[4] = {(cuuint64_t)d.stride, (cuuint64_t)d.numz, (cuuint64_t)d.numw,
                                    (cuuint64_t)p->batch};
        const cuuint64_t strides[3] = {4ull * d.stride, 4ull * d.stride * d.numz,
                                       4ull * (cuuint64_t)d.plane_size};
        const cuuint32_t box[4] = {(cuuint32_t)T->W[s], (cuuint32_t)T->Z[s], 1, 1};
        const cuuint32_t estr[4] = {1, 1, 1, 1};
        const CUresult r = enc(&T->map[s], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                               (void *)(p->d_planes + d.plane_off), dims, strides, box, estr,
                               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS)
            return fail(JERK_ECUDA, "cuTensorMapEncodeTiled failed for a volume tensor map");
    }
    p->tma = std::move(T);
    return JERK_OK;
}

extern "C" int jerk_plan_create(jerk_plan **out, const jerk_obs *obs, const jerk_subharm *subs,
                                int nsubs, const jerk_config *cfg)
{
    if (!out || !obs || !subs)
        return fail(JERK_EINVAL, "jerk_plan_create: null argument");
    *out = nullptr;
    if (obs->numharmstages < 1 || obs->numharmstages > kMaxStages ||
        nsubs != jerk_subharm_count(obs->numharmstages))
        return fail(JERK_EINVAL, "jerk_plan_create: nsubs does not match numharmstages");
    if (obs->norm_type != 0 && obs->norm_type != 1 && !(obs->nph > 0.0f))
        return fail(JERK_EINVAL, "norm_type must be 0 (block median) or 1 (local power)");
    if (obs->corr_uselen <= 0 || obs->corr_uselen % 2 || obs->corr_uselen > 65535)
        return fail(JERK_EINVAL, "bad corr_uselen");
    for (int s = 0; s < nsubs; s++)  // before any device work
        if (!fftlen_supported(subs[s].fftlen))
            return fail(JERK_EUNSUPPORTED, "unsupported fftlen " + std::to_string(subs[s].fftlen) +
                                               " (at most 15360 here)");

    jerk_plan *p = new jerk_plan();
    cudaGetDevice(&p->device);
    p->obs = *obs;
    p->nsubs = nsubs;
    p->subs.assign(subs, subs + nsubs);
    p->batch = (cfg && cfg->batch_rsteps > 0) ? cfg->batch_rsteps : 8;
    const int hm = cfg ? cfg->harm_mode : 0;
    if (hm < 0 || hm > 4) {
        delete p;
        return fail(JERK_EINVAL, "jerk_plan_create: harm_mode must be 0 .. 4");
    }
    // default: plain gathers, measured fastest at the paper configuration
    // (57.3 us per rstep against 69.6 with L2 prefetch and 93.7 with 16-row
    // TMA tiles)
    p->harm_mode = hm == 0 ? 1 : hm;
    p->harm_tile = p->harm_mode == 3 ? 8 : 16;
    p->use_graph = cfg && cfg->use_graph;
    const long long want_hits = (cfg && cfg->max_hits > 0) ? cfg->max_hits : (1LL << 22);
    if (cfg && cfg->stream) {
        p->stream = (cudaStream_t)cfg->stream;
    } else {
        cudaError_t e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            delete p;
            return cuda_fail(e, "cudaStreamCreate");
        }
        p->own_stream = true;
    }
    auto bail = [&](int code) {
        jerk_plan_destroy(p);
        return code;
    };

    const jerk_subharm &f = subs[0];
    if (f.numharm != 1 || f.harmnum != 1 || f.numz != obs->numz)
        return bail(fail(JERK_EINVAL, "subharmonic 0 must be the fundamental (1/1)"));
    p->zlo0 = calc_required_z(1.0, obs->zlo);
    p->wlo0 = calc_required_w(1.0, obs->wlo);
    p->nrsteps = count_rsteps(*obs);

    // steps: rlo / numrs of every (rstep, subharmonic)
    p->hsteps.resize((size_t)p->nrsteps * nsubs);
    std::vector<int> maxnumrs(nsubs, 0);
    const int rstep = (int)(obs->corr_uselen * kDR);
    for (long long k = 0; k < p->nrsteps; k++) {
        const double startr = obs->rlo + (double)k * rstep;
        const double lastr = startr + rstep - kDR;
        for (int s = 0; s < nsubs; s++) {
            const double hf = (double)subs[s].harmnum / (double)subs[s].numharm;
            const double drlo = calc_required_r(hf, startr), drhi = calc_required_r(hf, lastr);
            StepDev &st = p->hsteps[(size_t)k * nsubs + s];
            st.rlo = (long long)floor(drlo);
            st.fullrlo = startr;
            int numrs = (int)((ceil(drhi) - floor(drlo)) * kRDR + kDblCorrect) + 1;
            if (s == 0)
                numrs = obs->corr_uselen;
            else if (numrs % kRDR)
                numrs = (numrs / kRDR + 1) * kRDR;
            st.numrs = numrs;
            st.pad = 0;
            maxnumrs[s] = std::max(maxnumrs[s], numrs);
        }
    }

    // The harmonic sum addresses one batch's volumes with 32-bit offsets, so
    // the rsteps per batch (a speed knob only) are capped to what fits: at
    // zmax 600, wmax 1200 one rstep's volumes already hold 1.6 G floats.
    {
        long long per_rstep = 0;
        for (int s = 0; s < nsubs; s++)
            per_rstep += (long long)subs[s].numw * subs[s].numz * ((maxnumrs[s] + 3) & ~3);
        const long long cap = per_rstep > 0 ? ((1LL << 32) - 1) / per_rstep : p->batch;
        if (cap < 1)
            return bail(fail(JERK_EUNSUPPORTED, "ffdot volumes of one rstep exceed 2^32 floats"));
        p->batch = (int)std::min<long long>(p->batch, cap);
    }

    // subharmonic layout
    p->hsubs.resize(nsubs);
    long long kern_off = 0, plane_off = 0, data_off = 0;
    int zinds_off = 0, wind_off = 0;
    std::vector<uint16_t> zinds;
    std::vector<int> wind;
    std::map<int, int> twoff;
    int twtotal = 0;
    for (int s = 0; s < nsubs; s++) {
        const jerk_subharm &sh = subs[s];
        if (!fftlen_supported(sh.fftlen))
            return bail(fail(JERK_EUNSUPPORTED, "unsupported fftlen " + std::to_string(sh.fftlen)));
        if (maxnumrs[s] + 2 * sh.halfwidth > sh.fftlen)
            return bail(fail(JERK_EINVAL, "fftlen too short for the good bins"));
        SubDev &d = p->hsubs[s];
        d.numharm = sh.numharm;
        d.harmnum = sh.harmnum;
        d.harm_fract = (double)sh.harmnum / (double)sh.numharm;
        d.numz = sh.numz;
        d.numw = sh.numw;
        d.fftlen = sh.fftlen;
        d.halfwidth = sh.halfwidth;
        d.stride = (maxnumrs[s] + 3) & ~3;
        d.zlo = calc_required_z(d.harm_fract, obs->zlo);
        d.wlo = calc_required_w(d.harm_fract, obs->wlo);
        d.pownorm = (float)(1.0 / (double)(sh.fftlen * sh.fftlen));
        if (!twoff.count(sh.fftlen)) {
            twoff[sh.fftlen] = twtotal;
            twtotal += fft_twiddle_size(sh.fftlen);
        }
        d.twoff = twoff[sh.fftlen];
        d.kern_off = kern_off;
        kern_off += (long long)sh.numw * sh.numz * sh.fftlen;
        d.plane_size = (long long)sh.numw * sh.numz * d.stride;
        d.plane_off = plane_off;
        plane_off += d.plane_size * p->batch;
        d.data_off = data_off;
        data_off += (long long)sh.fftlen * p->batch;
        d.zinds_off = zinds_off;
        d.wind_off = wind_off;
        // zinds (src/accel_utils.c:1124-1130) and wind (src/accel_utils.c:1362-1364)
        for (int ii = 0; ii < obs->numz; ii++) {
            const double zz = obs->zlo + ii * kDZ;
            const int subz = calc_required_z(d.harm_fract, zz);
            const int zi = index_from_z(subz, d.zlo);
            if (s > 0 && (zi < 0 || zi >= sh.numz))
                return bail(fail(JERK_EINVAL, "zinds out of range"));
            zinds.push_back((uint16_t)zi);
        }
        for (int ii = 0; ii < subs[0].numw; ii++) {
            const int ww = p->wlo0 + ii * kDW;
            const int subw = calc_required_w(d.harm_fract, ww);
            const int wi = index_from_w(subw, d.wlo);
            if (s > 0 && (wi < 0 || wi >= sh.numw))
                return bail(fail(JERK_EINVAL, "wind out of range"));
            wind.push_back(wi);
        }
        zinds_off += obs->numz;
        wind_off += subs[0].numw;
        p->maxfft = std::max(p->maxfft, sh.fftlen);
        p->groups[sh.fftlen].push_back(s);
    }
    p->plane_floats = plane_off;
    p->prepped_f2 = data_off;
    if (plane_off >= (1LL << 32))
        return bail(fail(JERK_EINVAL, "ffdot volumes of one batch exceed 2^32 floats: lower batch_rsteps"));

    // twiddles: exp(-2 pi i m / N), double on the host
    std::vector<float2> tw;
    {
        std::vector<std::pair<int, int>> byoff;
        for (auto &kv : twoff)
            byoff.push_back({kv.second, kv.first});
        std::sort(byoff.begin(), byoff.end());
        for (auto &o : byoff)
            append_twiddles(o.second, tw);
    }
    for (int f = 0; f < 2; f++) {
        const int N = kFoldLens[f];
        if (!p->groups.count(N))
            continue;
        twtotal += twtotal & 1;  // 16-byte aligned tables
        p->fold_twoff[f] = twtotal;
        tw.resize(twtotal + fold_twiddle_size(N));
        fold_twiddle_table(N, tw.data() + twtotal);
        twtotal += fold_twiddle_size(N);
    }

#define JERK_CUDA_B(call)                                \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess)                           \
            return bail(cuda_fail(e_, #call));           \
    } while (0)

    // kernel bank
    if (cfg && cfg->device_bank) {
        p->d_bank = (float2 *)cfg->device_bank;
        p->own_bank = false;
    } else {
        JERK_CUDA_B(cudaMalloc(&p->d_bank, sizeof(float2) * kern_off));
        p->own_bank = true;
        for (int s = 0; s < nsubs; s++) {
            if (!subs[s].kernels)
                return bail(fail(JERK_EINVAL, "subharmonic without kernels and no device bank"));
            const size_t n = (size_t)subs[s].numw * subs[s].numz * subs[s].fftlen;
            JERK_CUDA_B(cudaMemcpyAsync(p->d_bank + p->hsubs[s].kern_off, subs[s].kernels,
                                        sizeof(float2) * n, cudaMemcpyHostToDevice, p->stream));
        }
    }
    JERK_CUDA_B(cudaMalloc(&p->d_tw, sizeof(float2) * twtotal));
    JERK_CUDA_B(cudaMemcpyAsync(p->d_tw, tw.data(), sizeof(float2) * twtotal,
                                cudaMemcpyHostToDevice, p->stream));
    // folded lengths: fold the bank's rows once for the half-length
    // correlation (the bank must be complete when the plan is made;
    // jerk_bank_generate returns once it is)
    std::vector<long long> fold_src[2];
    // device copies of the source-row tables, freed when this function
    // returns on any path (cudaFree waits for the fold kernels reading them)
    struct FoldSrc {
        long long *d[2] = {nullptr, nullptr};
        ~FoldSrc()
        {
            cudaFree(d[0]);
            cudaFree(d[1]);
        }
    } d_fold_src;
    for (int f = 0; f < 2; f++) {
        const int N = kFoldLens[f];
        if (p->fold_twoff[f] < 0)
            continue;
        for (int s : p->groups[N]) {
            const long long nrow = (long long)subs[s].numw * subs[s].numz;
            for (long long r = 0; r < nrow; r++)
                fold_src[f].push_back(p->hsubs[s].kern_off + r * N);
        }
        p->fold_floats2[f] = (long long)fold_src[f].size() * N;
        JERK_CUDA_B(cudaMalloc(&p->d_fold[f], sizeof(float2) * p->fold_floats2[f]));
        JERK_CUDA_B(cudaMalloc(&d_fold_src.d[f], sizeof(long long) * fold_src[f].size()));
        JERK_CUDA_B(cudaMemcpyAsync(d_fold_src.d[f], fold_src[f].data(),
                                    sizeof(long long) * fold_src[f].size(), cudaMemcpyHostToDevice,
                                    p->stream));
        JERK_CUDA_B(launch_fold_rows(N, p->d_bank, d_fold_src.d[f], p->d_fold[f],
                                     (int)fold_src[f].size(), p->stream));
    }
    JERK_CUDA_B(cudaMalloc(&p->d_subs, sizeof(SubDev) * nsubs));
    JERK_CUDA_B(cudaMemcpyAsync(p->d_subs, p->hsubs.data(), sizeof(SubDev) * nsubs,
                                cudaMemcpyHostToDevice, p->stream));
    if (p->nrsteps > 0) {
        JERK_CUDA_B(cudaMalloc(&p->d_steps, sizeof(StepDev) * p->hsteps.size()));
        JERK_CUDA_B(cudaMemcpyAsync(p->d_steps, p->hsteps.data(),
                                    sizeof(StepDev) * p->hsteps.size(), cudaMemcpyHostToDevice,
                                    p->stream));
    }
    JERK_CUDA_B(cudaMalloc(&p->d_zinds, sizeof(uint16_t) * zinds.size()));
    JERK_CUDA_B(cudaMemcpyAsync(p->d_zinds, zinds.data(), sizeof(uint16_t) * zinds.size(),
                                cudaMemcpyHostToDevice, p->stream));
    JERK_CUDA_B(cudaMalloc(&p->d_wind, sizeof(int) * wind.size()));
    JERK_CUDA_B(cudaMemcpyAsync(p->d_wind, wind.data(), sizeof(int) * wind.size(),
                                cudaMemcpyHostToDevice, p->stream));
    JERK_CUDA_B(cudaMalloc(&p->d_prepped, sizeof(float2) * p->prepped_f2));
    // one volume / rinds buffer: every launch of a pass runs on the plan's
    // stream, so batch k + 1's correlation starts after batch k's harmonic
    // sum has read the volumes (running the two side by side on two streams
    // measured slower than back to back: their CTAs then share SMs)
    JERK_CUDA_B(cudaMalloc(&p->d_planes, sizeof(float) * p->plane_floats));
    JERK_CUDA_B(cudaMalloc(&p->d_rinds, sizeof(uint16_t) * (size_t)p->batch * nsubs *
                                            obs->corr_uselen));
    if (p->harm_mode >= 2) {
        const int rc = build_harm_tma(p, p->harm_mode >= 3);
        if (rc != JERK_OK)
            return bail(rc);
        if (!p->tma)
            p->harm_mode = 1;  // no tensor maps here: the plain gather kernel
    }
    JERK_CUDA_B(cudaEventCreateWithFlags(&p->ev_done, cudaEventDisableTiming));
    for (int i = 0; i < jerk_plan::kRing; i++)
        JERK_CUDA_B(cudaEventCreateWithFlags(&p->ev_batch[i], cudaEventDisableTiming));
    JERK_CUDA_B(cudaHostAlloc(&p->h_counts, 2 * sizeof(unsigned int), cudaHostAllocDefault));
    JERK_CUDA_B(cudaMalloc(&p->d_hit_count, sizeof(unsigned int)));
    JERK_CUDA_B(cudaMalloc(&p->d_status, sizeof(unsigned int)));
    JERK_CUDA_B(cudaMemsetAsync(p->d_status, 0, sizeof(unsigned int), p->stream));
    {
        int rc = alloc_hits(p, want_hits);
        if (rc != JERK_OK)
            return bail(rc);
    }
    JERK_CUDA_B(cudaStreamSynchronize(p->stream));
#undef JERK_CUDA_B
    *out = p;
    return JERK_OK;
}

static int stage_spectrum(jerk_plan *p, const void *spectrum, int on_device, const float2 **spec)
{
    if (on_device && !p->use_graph) {
        *spec = (const float2 *)spectrum;
        return JERK_OK;
    }
    if (p->spec_cap < p->obs.numbins) {
        cudaFree(p->d_spec);
        p->d_spec = nullptr;
        JERK_CUDA(cudaMalloc(&p->d_spec, sizeof(float2) * p->obs.numbins));
        p->spec_cap = p->obs.numbins;
    }
    JERK_CUDA(cudaMemcpyAsync(p->d_spec, spectrum, sizeof(float2) * p->obs.numbins,
                              on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                              p->stream));
    if (!on_device)
        p->h2d_bytes += (long long)sizeof(float2) * p->obs.numbins;
    *spec = p->d_spec;
    return JERK_OK;
}

static SearchDev make_args(const jerk_plan *p, const float2 *spec)
{
    SearchDev a{};
    a.spec = spec;
    a.numbins = p->obs.numbins;
    a.lobin = p->obs.lobin;
    a.nsubs = p->nsubs;
    a.nstages = p->obs.numharmstages;
    a.corr_uselen = p->obs.corr_uselen;
    a.numz0 = p->subs[0].numz;
    a.numw0 = p->subs[0].numw;
    a.norm_type = p->obs.norm_type;
    a.nph = p->obs.nph;
    for (int i = 0; i < kMaxStages; i++)
        a.powcut[i] = i < p->obs.numharmstages ? p->obs.powcut[i] : INFINITY;
    a.subs = p->d_subs;
    a.steps = p->d_steps;
    a.bank = p->d_bank;
    a.twiddles = p->d_tw;
    a.zinds = p->d_zinds;
    a.wind = p->d_wind;
    a.prepped = p->d_prepped;
    a.planes = p->d_planes;
    a.rinds = p->d_rinds;
    a.hit_keys = p->d_hit_keys;
    a.hit_pows = p->d_hit_pows;
    a.hit_count = p->d_hit_count;
    a.max_hits = p->max_hits;
    a.status = p->d_status;
    return a;
}

// prep + correlation for one batch (volumes only)
static inline double fft_flops(int n)
{
    return 5.0 * n * log2((double)n);
}

// The plan's own correlation launch for one FFT length (the folded form at
// the folded lengths).
static cudaError_t launch_corr_of(const jerk_plan *p, const SearchDev &a, int N, const RowGroup &G,
                                  cudaStream_t st)
{
    const int f = fold_slot(N);
    if (f >= 0 && p->d_fold[f])
        return launch_corr_fold(N, a, G, G.rowstart[G.n], p->d_fold[f], p->d_tw + p->fold_twoff[f],
                                st);
    return launch_corr(a, N, G, G.rowstart[G.n], st);
}

// The rows of the subharmonics subs (one fftlen), numbered consecutively.
static RowGroup row_group(const jerk_plan *p, const std::vector<int> &subs)
{
    RowGroup G{};
    G.n = (int)subs.size();
    int rows = 0;
    for (int i = 0; i < G.n; i++) {
        const int s = subs[i];
        G.sub[i] = s;
        G.rowstart[i] = rows;
        rows += p->subs[s].numw * p->subs[s].numz;
    }
    G.rowstart[G.n] = rows;
    return G;
}

static int run_volumes(jerk_plan *p, SearchDev &a)
{
    {
        double bytes = 0, flops = 0;
        for (int s = 0; s < p->nsubs; s++) {
            const int N = p->subs[s].fftlen;
            bytes += (double)a.nb * (N / 2 * 8.0 + N / 2 * 8.0);
            flops += (double)a.nb * fft_flops(N);
        }
        const int tok = launch_begin(p, kclass(p, "prep"), bytes, flops);
        cudaError_t e = launch_prep(a, p->maxfft, p->stream);
        launch_end(p, tok);
        if (e != cudaSuccess)
            return cuda_fail(e, "prep_kernel");
    }
    cudaError_t e = cudaSuccess;
    for (auto &kv : p->groups) {
        const RowGroup G = row_group(p, kv.second);
        // algorithmic traffic: each kernel row read once per batch, each
        // prepared chunk read once, every good power written once
        const int N = kv.first;
        double bytes = 0, flops = 0;
        for (int i = 0; i < G.n; i++) {
            const int s = G.sub[i];
            const double nrow = (double)p->subs[s].numw * p->subs[s].numz;
            double numrs = 0;
            for (int b = 0; b < a.nb; b++)
                numrs += p->hsteps[(size_t)(a.first_rstep + b) * p->nsubs + s].numrs;
            bytes += nrow * N * 8.0 + a.nb * N / 2 * 8.0 + nrow * numrs * 4.0;
            flops += nrow * a.nb * (fft_flops(N) + 6.0 * N) + nrow * numrs * 3.0;
        }
        const int tok = launch_begin(p, kclass(p, "corr_" + std::to_string(N)), bytes, flops);
        e = launch_corr_of(p, a, N, G, p->stream);
        launch_end(p, tok);
        if (e != cudaSuccess)
            return cuda_fail(e, "corr_kernel");
    }
    return JERK_OK;
}

// A search pass is enqueued batch by batch, so a host thread driving several
// plans can keep each a few batches ahead of the device instead of filling
// the launch queue with one whole spectrum.

static int pass_begin(jerk_plan *p, const float2 *spec, long long first, long long count)
{
    jerk_plan::Pass &ps = p->pass;
    ps = jerk_plan::Pass();
    ps.a = make_args(p, spec);
    ps.first = first;
    ps.count = count;
    ps.next = first;
    JERK_CUDA(cudaMemsetAsync(p->d_hit_count, 0, sizeof(unsigned int), p->stream));
    // a pass that reported a failed wait or index leaves no trace in the next
    JERK_CUDA(cudaMemsetAsync(p->d_status, 0, sizeof(unsigned int), p->stream));
    if (p->wait_probe)
        JERK_CUDA(launch_wait_probe(p->d_status, p->stream));
    return JERK_OK;
}

// Batches whose harmonic sums have finished (non-blocking).
static long long pass_done_batches(jerk_plan *p)
{
    jerk_plan::Pass &ps = p->pass;
    while (ps.ndone < ps.nbatch && cudaEventQuery(p->ev_batch[ps.ndone % jerk_plan::kRing]) ==
                                       cudaSuccess)
        ps.ndone++;
    return ps.ndone;
}

// The plan's own harmonic-sum launch for batch arguments a.
static cudaError_t launch_harmsum_of(const jerk_plan *p, const SearchDev &a, cudaStream_t st)
{
    static const HarmTma no_maps{};
    return p->harm_mode >= 3 ? launch_harmsum_tma(a, *p->tma, p->harm_tile, st)
           : p->harm_mode == 2 ? launch_harmsum(a, *p->tma, true, st)
                               : launch_harmsum(a, no_maps, false, st);
}

// algorithmic traffic of one batch's harmonic sum: every volume read once
static void harmsum_work(const jerk_plan *p, const SearchDev &a, double *bytes, double *flops)
{
    double b = 0;
    const double npts = (double)a.nb * p->subs[0].numw * p->subs[0].numz * p->obs.corr_uselen;
    for (int s = 0; s < p->nsubs; s++) {
        double numrs = 0;
        for (int k = 0; k < a.nb; k++)
            numrs += p->hsteps[(size_t)(a.first_rstep + k) * p->nsubs + s].numrs;
        b += (double)p->subs[s].numw * p->subs[s].numz * numrs * 4.0;
    }
    *bytes += b;
    *flops += npts * p->nsubs;
}

static int pass_enqueue_one(jerk_plan *p)
{
    jerk_plan::Pass &ps = p->pass;
    SearchDev &a = ps.a;
    const long long k = ps.next;
    a.first_rstep = k;
    a.nb = (int)std::min<long long>(p->batch, ps.first + ps.count - k);
    a.planes = p->d_planes;
    a.rinds = p->d_rinds;
    int rc = run_volumes(p, a);
    if (rc != JERK_OK)
        return rc;
    double bytes = 0, flops = 0;
    harmsum_work(p, a, &bytes, &flops);
    const int tok = launch_begin(p, kclass(p, "harmsum"), bytes, flops);
    cudaError_t e = launch_harmsum_of(p, a, p->stream);
    launch_end(p, tok);
    if (e != cudaSuccess)
        return cuda_fail(e, "harmsum_kernel");
    if (!ps.capturing)
        JERK_CUDA(cudaEventRecord(p->ev_batch[ps.nbatch % jerk_plan::kRing], p->stream));
    ps.next += a.nb;
    ps.nbatch++;
    return JERK_OK;
}

static int pass_finish_enqueue(jerk_plan *p)
{
    jerk_plan::Pass &ps = p->pass;
    JERK_CUDA(cudaMemcpyAsync(p->h_counts, p->d_hit_count, sizeof(unsigned int),
                              cudaMemcpyDeviceToHost, p->stream));
    JERK_CUDA(cudaMemcpyAsync(p->h_counts + 1, p->d_status, sizeof(unsigned int),
                              cudaMemcpyDeviceToHost, p->stream));
    // (inside a capture an event record is only a dependency marker; graph
    // mode records ev_done after each launch of the graph instead)
    if (!ps.capturing)
        JERK_CUDA(cudaEventRecord(p->ev_done, p->stream));
    ps.all_enqueued = true;
    return JERK_OK;
}

// Enqueue batches until `ahead` of them are queued or running beyond those
// finished (ahead <= 0: all of them).  Returns 1 while batches remain to be
// enqueued, 0 once the pass is fully enqueued, < 0 on error.
static int pass_advance(jerk_plan *p, int ahead)
{
    jerk_plan::Pass &ps = p->pass;
    if (ps.error)
        return ps.error;
    if (ps.all_enqueued)
        return 0;
    const int limit = ahead <= 0 ? 1 << 30 : std::min(ahead, jerk_plan::kRing - 2);
    while (ps.next < ps.first + ps.count) {
        if (!ps.capturing && ps.nbatch - pass_done_batches(p) >= limit)
            return 1;
        int rc = pass_enqueue_one(p);
        if (rc != JERK_OK)
            return ps.error = rc;
    }
    int rc = pass_finish_enqueue(p);
    if (rc != JERK_OK)
        ps.error = rc;
    return rc == JERK_OK ? 0 : rc;
}

// Enqueue one whole search pass (no host synchronisation beyond the
// bookkeeping of pass_advance).
static int enqueue_search_pass(jerk_plan *p, const float2 *spec, long long first, long long count)
{
    int rc = pass_begin(p, spec, first, count);
    if (rc != JERK_OK)
        return rc;
    rc = pass_advance(p, 0);
    return rc < 0 ? rc : JERK_OK;
}

// Wait for an enqueued pass and read its hit count.
static int finish_search_pass(jerk_plan *p, unsigned int *nhits_out)
{
    JERK_CUDA(cudaEventSynchronize(p->ev_done));
    collect_timings(p);
    p->d2h_bytes += 2 * sizeof(unsigned int);
    if (p->h_counts[1] & 2u)
        return fail(JERK_ECUDA, "correlation: a data-row copy into shared memory timed out");
    if (p->h_counts[1])
        return fail(JERK_EINVAL, "harmonic sum: a subharmonic r index left its row");
    *nhits_out = p->h_counts[0];
    return JERK_OK;
}

static int run_search_pass(jerk_plan *p, const float2 *spec, long long first, long long count,
                           unsigned int *nhits_out)
{
    int rc = enqueue_search_pass(p, spec, first, count);
    if (rc != JERK_OK)
        return rc;
    return finish_search_pass(p, nhits_out);
}

static int check_range(const jerk_plan *p, long long first_rstep, long long num_rsteps,
                       long long *count)
{
    if (first_rstep < 0 || first_rstep > p->nrsteps)
        return fail(JERK_EINVAL, "jerk_search: first_rstep out of range");
    *count = p->nrsteps - first_rstep;
    if (num_rsteps > 0 && num_rsteps < *count)
        *count = num_rsteps;
    return JERK_OK;
}

// Graph mode: the first pass over (first, count) is captured from the plan's
// stream into a CUDA graph (every batch's prep, correlation and harmonic-sum
// launches, the hit-count read-back and the completion event) and replayed
// for every later spectrum; the spectrum is staged into d_spec beforehand, so
// the graph's pointers never change.  A hit-buffer reallocation drops it.
static int launch_graph_pass(jerk_plan *p, const float2 *spec, long long first, long long count)
{
    jerk_plan::Pass &ps = p->pass;
    if (!p->graph_exec || p->graph_first != first || p->graph_count != count) {
        drop_graph(p);
        JERK_CUDA(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
        int rc = pass_begin(p, spec, first, count);
        ps.capturing = true;
        if (rc == JERK_OK)
            rc = pass_advance(p, 0);
        cudaGraph_t g = nullptr;
        const cudaError_t ec = cudaStreamEndCapture(p->stream, &g);
        ps.capturing = false;
        if (rc < 0 || ec != cudaSuccess) {
            if (g)
                cudaGraphDestroy(g);
            ps.error = rc < 0 ? rc : JERK_ECUDA;
            return rc < 0 ? rc : cuda_fail(ec, "cudaStreamEndCapture");
        }
        const cudaError_t ei = cudaGraphInstantiate(&p->graph_exec, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
            p->graph_exec = nullptr;
            return cuda_fail(ei, "cudaGraphInstantiate");
        }
        p->graph_first = first;
        p->graph_count = count;
    }
    // the host bookkeeping of a fully enqueued pass
    ps = jerk_plan::Pass();
    ps.a = make_args(p, spec);
    ps.first = first;
    ps.count = count;
    ps.next = first + count;
    ps.all_enqueued = true;
    JERK_CUDA(cudaGraphLaunch(p->graph_exec, p->stream));
    JERK_CUDA(cudaEventRecord(p->ev_done, p->stream));
    p->graph_replays++;
    return JERK_OK;
}

extern "C" int jerk_search_async(jerk_plan *p, const void *spectrum, int spectrum_on_device,
                                 long long first_rstep, long long num_rsteps)
{
    if (!p || !spectrum)
        return fail(JERK_EINVAL, "jerk_search_async: null argument");
    if (p->in_flight)
        return fail(JERK_EINVAL, "jerk_search_async: a search is already in flight on this plan");
    long long count = 0;
    int rc = check_range(p, first_rstep, num_rsteps, &count);
    if (rc != JERK_OK)
        return rc;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != p->device)
        JERK_CUDA(cudaSetDevice(p->device));
    const float2 *spec = nullptr;
    rc = stage_spectrum(p, spectrum, spectrum_on_device, &spec);
    if (rc != JERK_OK)
        return rc;
    if (p->use_graph && !p->profiling) {
        rc = launch_graph_pass(p, spec, first_rstep, count);
    } else {
        rc = pass_begin(p, spec, first_rstep, count);
        if (rc == JERK_OK)
            rc = pass_advance(p, 4);
    }
    if (rc < 0)
        return rc;
    p->in_flight = true;
    p->inflight_spec = spec;
    p->inflight_first = first_rstep;
    p->inflight_count = count;
    return JERK_OK;
}

extern "C" int jerk_search_advance(jerk_plan *p, int ahead)
{
    if (!p || !p->in_flight)
        return 0;
    return pass_advance(p, ahead);
}

extern "C" int jerk_search_ready(jerk_plan *p)
{
    if (!p || !p->in_flight)
        return 1;
    if (p->pass.error)
        return p->pass.error;
    if (!p->pass.all_enqueued)
        return 0;
    const cudaError_t e = cudaEventQuery(p->ev_done);
    if (e == cudaSuccess)
        return 1;
    if (e == cudaErrorNotReady)
        return 0;
    return cuda_fail(e, "jerk_search_ready");
}

// ---------------------------------------------------------------------------
// Waves: the current batches of several plans' passes in merged launches --
// one prep launch, one correlation launch per FFT length and one harmonic
// sum per stage count, each covering every plan of the wave (up to
// kMaxGroupPlans) -- so spectra of uneven length and geometry share launches
// and small ones fill the GPU together.  Every plan's CTAs run as in its own
// launches, so its results are bitwise the same.

extern "C" int jerk_search_begin(jerk_plan *p, const void *spectrum, int spectrum_on_device,
                                 long long first_rstep, long long num_rsteps)
{
    if (!p || !spectrum)
        return fail(JERK_EINVAL, "jerk_search_begin: null argument");
    if (p->in_flight)
        return fail(JERK_EINVAL, "jerk_search_begin: a search is already in flight on this plan");
    long long count = 0;
    int rc = check_range(p, first_rstep, num_rsteps, &count);
    if (rc != JERK_OK)
        return rc;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != p->device)
        JERK_CUDA(cudaSetDevice(p->device));
    const float2 *spec = nullptr;
    rc = stage_spectrum(p, spectrum, spectrum_on_device, &spec);
    if (rc == JERK_OK)
        rc = pass_begin(p, spec, first_rstep, count);
    if (rc != JERK_OK)
        return rc;
    p->in_flight = true;
    p->inflight_spec = spec;
    p->inflight_first = first_rstep;
    p->inflight_count = count;
    return JERK_OK;
}

// One wave over W (same stream): every plan's next batch.
static int enqueue_wave(const std::vector<jerk_plan *> &W)
{
    jerk_plan *p0 = W[0];
    cudaStream_t st = p0->stream;
    const int n = (int)W.size();
    int maxfft = 0;
    double pbytes = 0, pflops = 0;
    for (jerk_plan *p : W) {
        jerk_plan::Pass &ps = p->pass;
        SearchDev &a = ps.a;
        a.first_rstep = ps.next;
        a.nb = (int)std::min<long long>(p->batch, ps.first + ps.count - ps.next);
        a.planes = p->d_planes;
        a.rinds = p->d_rinds;
        maxfft = std::max(maxfft, p->maxfft);
        for (int s = 0; s < p->nsubs; s++) {
            const int N = p->subs[s].fftlen;
            pbytes += (double)a.nb * (N / 2 * 8.0 + N / 2 * 8.0);
            pflops += (double)a.nb * fft_flops(N);
        }
    }
    auto fail_all = [&](cudaError_t e, const char *what) {
        const int rc = cuda_fail(e, what);
        for (jerk_plan *p : W)
            p->pass.error = rc;
        return rc;
    };
    GroupLaunch M{};
    M.n = n;
    for (int i = 0; i < n; i++)
        M.P[i] = W[i]->pass.a;
    int tok = launch_begin(p0, kclass(p0, "wave_prep"), pbytes, pflops);
    cudaError_t e = launch_prep_group(M, maxfft, st);
    launch_end(p0, tok);
    if (e != cudaSuccess)
        return fail_all(e, "prep_group_kernel");

    // correlation: one launch per FFT length over every plan that has it; a
    // plan whose rows of that length fill the GPU twice over by themselves
    // gains nothing from merging and takes its own (faster) launch
    std::map<int, std::vector<int>> byN;
    for (int i = 0; i < n; i++) {
        jerk_plan *p = W[i];
        for (auto &kv : p->groups) {
            const RowGroup G = row_group(p, kv.second);
            if (G.rowstart[G.n] < 2 * corr_wave_ctas(kv.first)) {
                byN[kv.first].push_back(i);
                continue;
            }
            tok = launch_begin(p0, kclass(p0, "wave_corr_" + std::to_string(kv.first)), 0.0, 0.0);
            e = launch_corr_of(p, p->pass.a, kv.first, G, st);
            launch_end(p0, tok);
            if (e != cudaSuccess)
                return fail_all(e, "corr_kernel");
        }
    }
    for (auto &kv : byN) {
        const int N = kv.first;
        GroupLaunch C{};
        C.n = (int)kv.second.size();
        double bytes = 0, flops = 0;
        const int f = fold_slot(N);
        bool fold = f >= 0;
        for (int j = 0; j < C.n; j++) {
            jerk_plan *p = W[kv.second[j]];
            const SearchDev &a = p->pass.a;
            C.P[j] = a;
            C.G[j] = row_group(p, p->groups.at(N));
            // at a folded length every plan has folded rows (made with the
            // plan), so the merged launch computes exactly what the plan's
            // own launch does
            fold = fold && p->d_fold[f];
            C.fold[j] = f >= 0 ? p->d_fold[f] : nullptr;
            C.fold_tw[j] = f >= 0 && p->d_fold[f] ? p->d_tw + p->fold_twoff[f] : nullptr;
            for (int g = 0; g < C.G[j].n; g++) {
                const int s = C.G[j].sub[g];
                const double nrow = (double)p->subs[s].numw * p->subs[s].numz;
                double numrs = 0;
                for (int b = 0; b < a.nb; b++)
                    numrs += p->hsteps[(size_t)(a.first_rstep + b) * p->nsubs + s].numrs;
                bytes += nrow * N * 8.0 + a.nb * N / 2 * 8.0 + nrow * numrs * 4.0;
                flops += nrow * a.nb * (fft_flops(N) + 6.0 * N) + nrow * numrs * 3.0;
            }
        }
        tok = launch_begin(p0, kclass(p0, "wave_corr_" + std::to_string(N)), bytes, flops);
        e = fold ? launch_corr_fold_group(N, C, st) : launch_corr_group(C, N, st);
        launch_end(p0, tok);
        if (e != cudaSuccess)
            return fail_all(e, "corr_group_kernel");
    }

    // harmonic sums: the gather form merged per stage count; plans tuned to
    // another form launch their own
    std::map<int, std::vector<int>> byS;
    for (int i = 0; i < n; i++) {
        jerk_plan *p = W[i];
        const SearchDev &a = p->pass.a;
        const long long ctas = (long long)((a.corr_uselen + 127) / 128) * a.numw0 * a.nb;
        if (p->harm_mode <= 1 && ctas < 2 * harmsum_wave_ctas(a.nstages)) {
            byS[p->obs.numharmstages].push_back(i);
            continue;
        }
        double bytes = 0, flops = 0;
        harmsum_work(p, p->pass.a, &bytes, &flops);
        tok = launch_begin(p0, kclass(p0, "wave_harmsum"), bytes, flops);
        e = launch_harmsum_of(p, p->pass.a, st);
        launch_end(p0, tok);
        if (e != cudaSuccess)
            return fail_all(e, "harmsum_kernel");
    }
    for (auto &kv : byS) {
        GroupLaunch H{};
        H.n = (int)kv.second.size();
        double bytes = 0, flops = 0;
        for (int j = 0; j < H.n; j++) {
            jerk_plan *p = W[kv.second[j]];
            H.P[j] = p->pass.a;
            harmsum_work(p, p->pass.a, &bytes, &flops);
        }
        tok = launch_begin(p0, kclass(p0, "wave_harmsum"), bytes, flops);
        e = launch_harmsum_group(H, kv.first, st);
        launch_end(p0, tok);
        if (e != cudaSuccess)
            return fail_all(e, "harmsum_group_kernel");
    }

    for (jerk_plan *p : W) {
        jerk_plan::Pass &ps = p->pass;
        JERK_CUDA(cudaEventRecord(p->ev_batch[ps.nbatch % jerk_plan::kRing], st));
        ps.next += ps.a.nb;
        ps.nbatch++;
        if (ps.next >= ps.first + ps.count) {
            const int rc = pass_finish_enqueue(p);
            if (rc != JERK_OK)
                return ps.error = rc;
        }
    }
    return JERK_OK;
}

extern "C" int jerk_group_advance(jerk_plan *const *plans, int nplans, int ahead)
{
    if (!plans || nplans < 0)
        return fail(JERK_EINVAL, "jerk_group_advance: bad argument");
    jerk_plan *first = nullptr;
    for (int i = 0; i < nplans; i++) {
        jerk_plan *p = plans[i];
        if (!p)
            return fail(JERK_EINVAL, "jerk_group_advance: null plan");
        if (!p->in_flight || p->pass.all_enqueued || p->pass.error)
            continue;
        if (!first)
            first = p;
        else if (p->stream != first->stream || p->device != first->device)
            return fail(JERK_EINVAL, "jerk_group_advance: plans on different streams or devices");
    }
    if (!first)
        return 0;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != first->device)
        JERK_CUDA(cudaSetDevice(first->device));
    const int limit = ahead <= 0 ? 1 << 30 : std::min(ahead, jerk_plan::kRing - 2);
    for (;;) {
        std::vector<jerk_plan *> sel;
        bool left = false;
        for (int i = 0; i < nplans; i++) {
            jerk_plan *p = plans[i];
            jerk_plan::Pass &ps = p->pass;
            if (!p->in_flight || ps.all_enqueued || ps.error)
                continue;
            left = true;
            if (ps.nbatch - pass_done_batches(p) < limit)
                sel.push_back(p);
        }
        if (sel.empty())
            return left ? 1 : 0;
        for (size_t i = 0; i < sel.size(); i += kMaxGroupPlans) {
            std::vector<jerk_plan *> W(sel.begin() + i,
                                       sel.begin() + std::min(sel.size(), i + kMaxGroupPlans));
            const int rc = enqueue_wave(W);
            if (rc != JERK_OK)
                return rc;
        }
    }
}

extern "C" int jerk_search_group(jerk_plan *const *plans, const void *const *spectra,
                                 const int *spectrum_on_device, int nplans, jerk_cand **cands,
                                 long long *ncands)
{
    if (!plans || !spectra || !spectrum_on_device || !cands || !ncands || nplans < 1)
        return fail(JERK_EINVAL, "jerk_search_group: bad argument");
    for (int i = 0; i < nplans; i++) {
        cands[i] = nullptr;
        ncands[i] = 0;
    }
    int rc = JERK_OK, began = 0;
    for (; began < nplans && rc == JERK_OK; began++)
        rc = jerk_search_begin(plans[began], spectra[began], spectrum_on_device[began], 0, 0);
    if (rc != JERK_OK)
        began--;  // the failed one holds no pass
    if (rc == JERK_OK)
        rc = jerk_group_advance(plans, nplans, 0);
    // every begun pass is collected (ends its in-flight state), even after a
    // failure; the first error is returned
    for (int i = 0; i < began; i++) {
        const int r = jerk_search_collect(plans[i], &cands[i], &ncands[i], nullptr);
        if (rc == JERK_OK)
            rc = r;
    }
    return rc;
}

// What decoding a hit key needs: the fundamental's geometry and, per rstep,
// the fundamental's first r (hsteps[rs][0].rlo).
struct HitGeom {
    int S = 1;
    long long numrs0 = 0, numz0 = 0, numw0 = 0;
    int zlo0 = 0, wlo0 = 0;
    const long long *numindep = nullptr;
    std::function<long long(long long)> rlo_of;
};

// Hits in key order -- the reference's insertion order (rstep, stage, w, z,
// r; src/accel_utils_cu.c:857-929) -- decoded into candidates with their
// sigma and inserted with the reference's rule.  order receives the sorted
// permutation of the input.
static void hits_to_list(const HitGeom &g, const unsigned long long *keys, const float *pows,
                         uint32_t nh, std::vector<uint32_t> &order, CandList &L)
{
    order.resize(nh);
    for (uint32_t i = 0; i < nh; i++)
        order[i] = i;
    std::sort(order.begin(), order.end(),
              [&](uint32_t x, uint32_t y) { return keys[x] < keys[y]; });
    // decode + sigma per hit (independent, so spread over host threads when
    // there are many), then the insertions in key order (sequential: each
    // depends on the list the earlier ones left)
    std::vector<jerk_cand> cv(nh);
    auto decode = [&](uint32_t lo, uint32_t hi) {
        for (uint32_t i = lo; i < hi; i++) {
            unsigned long long key = keys[order[i]];
            const int kk = (int)(key % g.numrs0);
            key /= g.numrs0;
            const int jj = (int)(key % g.numz0);
            key /= g.numz0;
            const int ii = (int)(key % g.numw0);
            key /= g.numw0;
            const int stage = (int)(key % g.S);
            const long long rs = (long long)(key / g.S);
            const int nhm = 1 << stage;
            jerk_cand &c = cv[i];
            c.power = pows[order[i]];
            c.sigma = (float)jerk_candidate_sigma(c.power, nhm, (double)g.numindep[stage]);
            c.numharm = nhm;
            c.r = ((double)g.rlo_of(rs) + kk * kDR) / (double)nhm;
            c.z = (g.zlo0 + jj * (double)kDZ) / (double)nhm;
            c.w = (g.wlo0 + ii * (double)kDW) / (double)nhm;
        }
    };
    const uint32_t nthr =
        nh < 8192 ? 1u : std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    if (nthr == 1) {
        decode(0, nh);
    } else {
        std::vector<std::thread> pool;
        const uint32_t per = (nh + nthr - 1) / nthr;
        for (uint32_t t = 0; t < nthr; t++) {
            const uint32_t lo = t * per, hi = std::min(nh, lo + per);
            if (lo < hi)
                pool.emplace_back(decode, lo, hi);
        }
        for (auto &th : pool)
            th.join();
    }
    for (uint32_t i = 0; i < nh; i++)
        insert_cand(L, cv[i]);
}

extern "C" int jerk_search_collect(jerk_plan *p, jerk_cand **cands, long long *ncands,
                                   jerk_hits *hits)
{
    if (!p || !p->in_flight)
        return fail(JERK_EINVAL, "jerk_search_collect: no search in flight");
    p->in_flight = false;
    unsigned int nh = 0;
    int rc = pass_advance(p, 0);  // whatever is not enqueued yet
    if (rc < 0) {
        cudaStreamSynchronize(p->stream);  // what was enqueued ends before the plan is reused
        return rc;
    }
    rc = finish_search_pass(p, &nh);
    if (rc != JERK_OK)
        return rc;
    for (int attempt = 0; (long long)nh > p->max_hits; attempt++) {
        // overflow: the counter kept counting, so one retry with the exact
        // size always suffices
        if (attempt > 2)
            return fail(JERK_OVERFLOW, "hit buffer overflow persisted");
        rc = alloc_hits(p, (long long)nh + (nh >> 3) + 1024);
        if (rc != JERK_OK)
            return rc;
        rc = run_search_pass(p, p->inflight_spec, p->inflight_first, p->inflight_count, &nh);
        if (rc != JERK_OK)
            return rc;
    }

    // hits back, in the reference's insertion order
    std::vector<unsigned long long> keys(nh);
    std::vector<float> pows(nh);
    if (nh) {
        // the pass has ended (ev_done); a synchronous copy does not wait for
        // other work queued behind it on a stream shared with other plans
        JERK_CUDA(cudaMemcpy(keys.data(), p->d_hit_keys, sizeof(unsigned long long) * nh,
                             cudaMemcpyDeviceToHost));
        JERK_CUDA(cudaMemcpy(pows.data(), p->d_hit_pows, sizeof(float) * nh,
                             cudaMemcpyDeviceToHost));
        p->d2h_bytes += (long long)nh * (sizeof(unsigned long long) + sizeof(float));
    }
    HitGeom g;
    g.S = p->obs.numharmstages;
    g.numrs0 = p->obs.corr_uselen;
    g.numz0 = p->subs[0].numz;
    g.numw0 = p->subs[0].numw;
    g.zlo0 = p->zlo0;
    g.wlo0 = p->wlo0;
    g.numindep = p->obs.numindep;
    g.rlo_of = [p](long long rs) { return p->hsteps[(size_t)rs * p->nsubs].rlo; };
    CandList L;
    std::vector<uint32_t> order;
    hits_to_list(g, keys.data(), pows.data(), nh, order, L);
    if (hits) {
        hits->count = nh;
        hits->keys = (unsigned long long *)malloc(sizeof(unsigned long long) * (nh ? nh : 1));
        hits->powers = (float *)malloc(sizeof(float) * (nh ? nh : 1));
        for (uint32_t i = 0; i < nh; i++) {
            hits->keys[i] = keys[order[i]];
            hits->powers[i] = pows[order[i]];
        }
    }
    const long long n = export_list(L, cands);
    if (n < 0)
        return fail(JERK_ENOMEM, "candidate list allocation");
    if (ncands)
        *ncands = n;
    return JERK_OK;
}

extern "C" int jerk_merge_hits(const jerk_obs *obs, const jerk_subharm *fundamental,
                               const unsigned long long *keys, const float *powers,
                               long long nhits, jerk_cand **cands, long long *ncands)
{
    if (!obs || !fundamental || !cands || nhits < 0 || (nhits && (!keys || !powers)))
        return fail(JERK_EINVAL, "jerk_merge_hits: bad argument");
    if (nhits > 0xffffffffll)
        return fail(JERK_EUNSUPPORTED, "jerk_merge_hits: more than 2^32 hits");
    if (fundamental->numharm != 1 || fundamental->harmnum != 1 || fundamental->numz != obs->numz ||
        fundamental->numw < 1 || obs->corr_uselen < 2 || obs->numharmstages < 1 ||
        obs->numharmstages > JERK_MAX_STAGES)
        return fail(JERK_EINVAL, "jerk_merge_hits: fundamental and obs do not match");
    const long long nrsteps = count_rsteps(*obs);
    const long long per_rstep = (long long)obs->numharmstages * fundamental->numw *
                                fundamental->numz * obs->corr_uselen;
    for (long long i = 0; i < nhits; i++)
        if (keys[i] / (unsigned long long)per_rstep >= (unsigned long long)nrsteps)
            return fail(JERK_EINVAL, "jerk_merge_hits: a key lies beyond the last rstep");
    HitGeom g;
    g.S = obs->numharmstages;
    g.numrs0 = obs->corr_uselen;
    g.numz0 = fundamental->numz;
    g.numw0 = fundamental->numw;
    g.zlo0 = calc_required_z(1.0, obs->zlo);
    g.wlo0 = calc_required_w(1.0, obs->wlo);
    g.numindep = obs->numindep;
    const int rstep = (int)(obs->corr_uselen * kDR);
    const double rlo = obs->rlo;
    // as the plan's step table: floor(calc_required_r(1, startr))
    g.rlo_of = [rstep, rlo](long long rs) {
        return (long long)floor(calc_required_r(1.0, rlo + (double)rs * rstep));
    };
    CandList L;
    std::vector<uint32_t> order;
    hits_to_list(g, keys, powers, (uint32_t)nhits, order, L);
    const long long n = export_list(L, cands);
    if (n < 0)
        return fail(JERK_ENOMEM, "candidate list allocation");
    if (ncands)
        *ncands = n;
    return JERK_OK;
}

extern "C" int jerk_search(jerk_plan *p, const void *spectrum, int spectrum_on_device,
                           long long first_rstep, long long num_rsteps, jerk_cand **cands,
                           long long *ncands, jerk_hits *hits)
{
    int rc = jerk_search_async(p, spectrum, spectrum_on_device, first_rstep, num_rsteps);
    if (rc != JERK_OK)
        return rc;
    return jerk_search_collect(p, cands, ncands, hits);
}

extern "C" long long jerk_plan_device_bytes(const jerk_plan *p)
{
    if (!p)
        return 0;
    return (long long)(sizeof(float) * p->plane_floats +
                       sizeof(uint16_t) * (size_t)p->batch * p->nsubs * p->obs.corr_uselen +
                       sizeof(float2) * p->prepped_f2 +
                       (sizeof(unsigned long long) + sizeof(float)) * p->max_hits +
                       sizeof(StepDev) * p->hsteps.size() + sizeof(float2) * p->spec_cap +
                       sizeof(float2) * (p->fold_floats2[0] + p->fold_floats2[1]) +
                       (p->own_bank ? sizeof(float2) * jerk_bank_elements(p->subs.data(), p->nsubs)
                                    : 0));
}

extern "C" int jerk_debug_wait_probe(jerk_plan *p, int on)
{
    if (!p)
        return fail(JERK_EINVAL, "jerk_debug_wait_probe: null plan");
    if (p->in_flight)
        return fail(JERK_EINVAL, "jerk_debug_wait_probe: a search is in flight");
    p->wait_probe = on != 0;
    drop_graph(p);  // a captured pass holds the old launch arguments
    return JERK_OK;
}

extern "C" int jerk_debug_volume(jerk_plan *p, const void *spectrum, int spectrum_on_device,
                                 long long rstep, int sub, float *out, int *numrs, long long *rlo)
{
    if (!p || !spectrum || !out || sub < 0 || sub >= p->nsubs || rstep < 0 ||
        rstep >= p->nrsteps)
        return fail(JERK_EINVAL, "jerk_debug_volume: bad argument");
    const float2 *spec = nullptr;
    int rc = stage_spectrum(p, spectrum, spectrum_on_device, &spec);
    if (rc != JERK_OK)
        return rc;
    SearchDev a = make_args(p, spec);
    a.first_rstep = rstep;
    a.nb = 1;
    rc = run_volumes(p, a);
    if (rc != JERK_OK)
        return rc;
    JERK_CUDA(cudaStreamSynchronize(p->stream));
    collect_timings(p);
    const SubDev &d = p->hsubs[sub];
    const StepDev &st = p->hsteps[(size_t)rstep * p->nsubs + sub];
    JERK_CUDA(cudaMemcpy2DAsync(out, sizeof(float) * st.numrs, p->d_planes + d.plane_off,
                                sizeof(float) * d.stride, sizeof(float) * st.numrs,
                                (size_t)d.numw * d.numz, cudaMemcpyDeviceToHost, p->stream));
    JERK_CUDA(cudaStreamSynchronize(p->stream));
    if (numrs)
        *numrs = st.numrs;
    if (rlo)
        *rlo = st.rlo;
    return JERK_OK;
}
