// The served form: a request loop on one GPU.
//
// Spectra arrive at any time (jerk_server_submit); a worker thread that owns
// the device admits them while slots and HBM allow (footprint = ffdot volumes
// + tables + hit buffer + the spectrum, plus the kernel bank if it is not
// already resident), keeps several searches in flight at once (continuous
// batching: a new request starts as soon as another one finishes and frees
// its slot), and hands finished candidate lists back through
// jerk_server_poll.  Kernel banks are generated on the GPU once per
// (zmax, wmax, numharm, geometry) and shared by every request that matches;
// idle plans with identical geometry are reused instead of reallocated.
//
// The active searches share one stream, and their work overlaps on the
// device: the worker enqueues waves (jerk_group_advance), each one merged
// launch per kernel kind over the next batch of every active search, a few
// waves ahead of the device.  A request admitted while others run joins the
// next wave.  (Kernels of different searches on separate streams sharing SMs
// measured slower than the same kernels in sequence; merged launches give
// the overlap without that contention.)
//
// It is built only on the public C ABI of jerk.h, so its results are exactly
// jerk_search's for the same spectrum and parameters, alone or in a mix.
// (The reference's counterpart is a process pool with one CPU1/GPU/CPU2
// thread triple per worker, bin/accelsearch_pipeline_cu.py:296-407.)
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "jerk.h"

namespace {

double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Geometry {
    jerk_obs obs;
    int fftlen = 0;
    std::vector<jerk_subharm> subs;
};

using BankKey = std::tuple<int, int, int, int, int>;  // zlo, wlo, stages, corr_uselen, fftlen

struct Bank {
    void *ptr = nullptr;
    long long bytes = 0;
    int users = 0;
    double last_used = 0;
};

struct Slot {
    jerk_request req;
    Geometry geo;
    BankKey key;
    jerk_plan *plan = nullptr;
    long long bytes = 0;
    double t_submit = 0, t_start = 0;
    void *series = nullptr;  // time-series requests: the series, then its spectrum, + scratch
    long long series_bytes = 0;
};

struct IdlePlan {
    jerk_plan *plan;
    jerk_obs obs;
    BankKey key;
    long long bytes;
};

struct SeriesBuf {
    void *ptr;
    long long bytes;
};

struct Pending {
    jerk_request req;
    double t_submit;
};

bool same_obs(const jerk_obs &a, const jerk_obs &b) { return memcmp(&a, &b, sizeof(a)) == 0; }

}  // namespace

struct jerk_server {
    jerk_server_config cfg{};
    cudaStream_t stream = nullptr;  // shared by every plan of this server
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stop = false;
    std::deque<Pending> pending;
    std::deque<jerk_result> done;
    // worker-owned
    std::vector<Slot> active;
    std::vector<IdlePlan> idle;
    std::vector<SeriesBuf> series_pool;  // time-series buffers between requests
    std::map<BankKey, Bank> banks;
    long long bytes_in_use = 0;
    // counters (under mu)
    long long submitted = 0, finished = 0, failed = 0;
    long long peak_bytes = 0;
    long long h2d_bytes = 0, d2h_bytes = 0;  // host<->device traffic of finished requests
};

static int geometry_of(const jerk_request &r, Geometry *g)
{
    int mk = 0;
    int rc = jerk_obs_from_params(r.numbins, r.N, r.dt, r.zmax, r.wmax, r.wmax_given, r.numharm,
                                  r.sigma, r.flo, r.fhi, &g->obs, &g->fftlen, &mk);
    if (rc != JERK_OK)
        return rc;
    const int n = jerk_subharm_count(g->obs.numharmstages);
    g->subs.resize(n);
    for (int i = 0; i < n; i++) {
        rc = jerk_subharm_sizes(&g->obs, g->fftlen, i, &g->subs[i]);
        if (rc != JERK_OK)
            return rc;
    }
    return JERK_OK;
}

static BankKey key_of(const Geometry &g)
{
    return BankKey((int)g.obs.zlo, (int)g.obs.wlo, g.obs.numharmstages, g.obs.corr_uselen,
                   g.fftlen);
}

// Device bytes a plan for g will hold (volumes, rinds, chunks, hit buffer,
// steps, spectrum staging, and its folded copy of the fftlen-2048 and -1280
// rows).
static long long plan_footprint(const Geometry &g, int batch)
{
    long long vol = 0, chunks = 0, folded = 0;
    for (const auto &s : g.subs) {
        const double hf = (double)s.harmnum / s.numharm;
        const long long stride = (((long long)(g.obs.corr_uselen * hf) + 8) + 3) & ~3LL;
        vol += (long long)s.numw * s.numz * stride * 4;
        chunks += (long long)s.fftlen * 8;
        if (s.fftlen == 2048 || s.fftlen == 1280)
            folded += (long long)s.numw * s.numz * s.fftlen * 8;
    }
    const long long rsteps = (long long)((g.obs.highestbin - g.obs.rlo) / (g.obs.corr_uselen / 2)) + 1;
    return vol * batch + chunks * batch +
           2LL * batch * (long long)g.subs.size() * g.obs.corr_uselen +
           (long long)(1 << 22) * 12 + rsteps * (long long)g.subs.size() * 24 +
           g.obs.numbins * 8 + folded + (64LL << 20);
}

// Device bytes of a time-series request's buffer: the series (turned into its
// spectrum in place), then the preparation's scratch.
static long long series_footprint(const jerk_request &r)
{
    if (!r.timeseries)
        return 0;
    return ((4 * r.N + 255) & ~255LL) + jerk_spectrum_scratch_bytes(r.N);
}

// Back to the pool (freeing would synchronise the device under the other
// searches); the stream orders its next use after everything that read it.
static void release_series(jerk_server *s, Slot &sl)
{
    if (sl.series) {
        s->series_pool.push_back(SeriesBuf{sl.series, sl.series_bytes});
        sl.series = nullptr;
        sl.series_bytes = 0;
    }
}

static bool pool_fits(const jerk_server *s, long long bytes)
{
    for (const auto &b : s->series_pool)
        if (b.bytes >= bytes)
            return true;
    return false;
}

// Upload (if on the host) and prepare a time-series request's spectrum on the
// server's stream, ahead of its search there.
static int prepare_series(jerk_server *s, Slot &sl)
{
    const long long bytes = series_footprint(sl.req);
    for (size_t i = 0; i < s->series_pool.size(); i++) {
        if (s->series_pool[i].bytes >= bytes) {
            sl.series = s->series_pool[i].ptr;
            sl.series_bytes = s->series_pool[i].bytes;
            s->series_pool.erase(s->series_pool.begin() + i);
            break;
        }
    }
    if (!sl.series) {
        const int rc = jerk_device_alloc(bytes, &sl.series);
        if (rc != JERK_OK)
            return rc;
        sl.series_bytes = bytes;
        s->bytes_in_use += bytes;
    }
    const long long sbytes = 4 * sl.req.N;
    const long long off = (sbytes + 255) & ~255LL;
    if (!sl.req.on_device) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->h2d_bytes += sbytes;
    }
    if (cudaMemcpyAsync(sl.series, sl.req.spectrum, (size_t)sbytes,
                        sl.req.on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                        s->stream) != cudaSuccess)
        return JERK_ECUDA;
    int rc = jerk_spectrum_from_timeseries((const float *)sl.series, sl.req.N, sl.series,
                                           (char *)sl.series + off, sl.series_bytes - off,
                                           s->stream);
    if (rc == JERK_OK && sl.req.numbirds > 0)
        rc = jerk_zap_birdies(sl.series, sl.req.N / 2, sl.req.N, sl.req.bird_lobins,
                              sl.req.bird_hibins, sl.req.numbirds, s->stream);
    return rc;
}

static void release_bank(jerk_server *s, const BankKey &k)
{
    auto it = s->banks.find(k);
    if (it != s->banks.end()) {
        it->second.users--;
        it->second.last_used = now_s();
    }
}

// Free idle plans and unused banks until `need` more bytes fit the budget.
static void make_room(jerk_server *s, long long need)
{
    while (s->bytes_in_use + need > s->cfg.hbm_budget_bytes && !s->series_pool.empty()) {
        jerk_device_free(s->series_pool.back().ptr);
        s->bytes_in_use -= s->series_pool.back().bytes;
        s->series_pool.pop_back();
    }
    while (s->bytes_in_use + need > s->cfg.hbm_budget_bytes && !s->idle.empty()) {
        IdlePlan ip = s->idle.front();
        s->idle.erase(s->idle.begin());
        jerk_plan_destroy(ip.plan);
        s->bytes_in_use -= ip.bytes;
    }
    while (s->bytes_in_use + need > s->cfg.hbm_budget_bytes) {
        auto victim = s->banks.end();
        for (auto it = s->banks.begin(); it != s->banks.end(); ++it)
            if (it->second.users == 0 &&
                (victim == s->banks.end() || it->second.last_used < victim->second.last_used))
                victim = it;
        if (victim == s->banks.end())
            break;
        jerk_device_free(victim->second.ptr);
        s->bytes_in_use -= victim->second.bytes;
        s->banks.erase(victim);
    }
}

static void finish(jerk_server *s, const jerk_request &req, double t_submit, double t_start,
                   int status, jerk_cand *cands, long long n)
{
    jerk_result r{};
    r.tag = req.tag;
    r.status = status;
    r.cands = cands;
    r.ncands = n;
    r.t_submit = t_submit;
    r.t_start = t_start;
    r.t_done = now_s();
    std::lock_guard<std::mutex> lk(s->mu);
    s->done.push_back(r);
    s->finished++;
    if (status != JERK_OK)
        s->failed++;
    s->cv_done.notify_all();
}

// Try to start one pending request; false if it has to wait for room.
static bool admit(jerk_server *s, const Pending &pd)
{
    Slot sl;
    sl.req = pd.req;
    sl.t_submit = pd.t_submit;
    int rc = geometry_of(pd.req, &sl.geo);
    if (rc != JERK_OK) {
        finish(s, pd.req, pd.t_submit, now_s(), rc, nullptr, 0);
        return true;
    }
    sl.key = key_of(sl.geo);
    // an idle plan with this exact geometry?
    for (size_t i = 0; i < s->idle.size(); i++) {
        if (s->idle[i].key == sl.key && same_obs(s->idle[i].obs, sl.geo.obs)) {
            sl.plan = s->idle[i].plan;
            sl.bytes = s->idle[i].bytes;
            s->idle.erase(s->idle.begin() + i);
            break;
        }
    }
    const bool have_bank = s->banks.count(sl.key) > 0;
    if (have_bank)
        s->banks[sl.key].users++;  // pinned while this request is admitted
    const long long bank_bytes =
        have_bank ? 0 : 8 * jerk_bank_elements(sl.geo.subs.data(), (int)sl.geo.subs.size());
    const long long series_bytes =
        pool_fits(s, series_footprint(pd.req)) ? 0 : series_footprint(pd.req);
    const long long need = (sl.plan ? 0 : plan_footprint(sl.geo, s->cfg.batch_rsteps)) + bank_bytes +
                           series_bytes;
    if (need > s->cfg.hbm_budget_bytes) {
        // can never fit, even alone: fail this request, keep serving the rest
        if (sl.plan)
            s->idle.push_back(IdlePlan{sl.plan, sl.geo.obs, sl.key, sl.bytes});
        if (have_bank)
            release_bank(s, sl.key);
        finish(s, pd.req, pd.t_submit, now_s(), JERK_ENOMEM, nullptr, 0);
        return true;
    }
    if (s->bytes_in_use + need > s->cfg.hbm_budget_bytes) {
        make_room(s, need);
        if (s->bytes_in_use + need > s->cfg.hbm_budget_bytes && !s->active.empty()) {
            if (sl.plan)
                s->idle.push_back(IdlePlan{sl.plan, sl.geo.obs, sl.key, sl.bytes});
            if (have_bank)
                release_bank(s, sl.key);
            return false;  // wait for a running search to free memory
        }
    }
    sl.t_start = now_s();
    if (!have_bank) {
        Bank b;
        b.bytes = bank_bytes;
        rc = jerk_device_alloc(b.bytes, &b.ptr);
        if (rc == JERK_OK)
            rc = jerk_bank_generate(sl.geo.subs.data(), (int)sl.geo.subs.size(), b.ptr, nullptr);
        if (rc != JERK_OK) {
            if (b.ptr)
                jerk_device_free(b.ptr);
            if (sl.plan)
                s->idle.push_back(IdlePlan{sl.plan, sl.geo.obs, sl.key, sl.bytes});
            finish(s, pd.req, pd.t_submit, sl.t_start, rc, nullptr, 0);
            return true;
        }
        b.users = 1;
        s->banks[sl.key] = b;
        s->bytes_in_use += b.bytes;
    }
    Bank &bank = s->banks[sl.key];
    if (!sl.plan) {
        jerk_config c{};
        c.batch_rsteps = s->cfg.batch_rsteps;
        c.harm_mode = s->cfg.harm_mode;
        c.device_bank = bank.ptr;
        c.stream = s->stream;
        rc = jerk_plan_create(&sl.plan, &sl.geo.obs, sl.geo.subs.data(), (int)sl.geo.subs.size(), &c);
        if (rc != JERK_OK) {
            release_bank(s, sl.key);
            finish(s, pd.req, pd.t_submit, sl.t_start, rc, nullptr, 0);
            return true;
        }
        sl.bytes = jerk_plan_device_bytes(sl.plan);
        s->bytes_in_use += sl.bytes;
    }
    if (pd.req.timeseries) {
        rc = prepare_series(s, sl);
        if (rc == JERK_OK)
            rc = jerk_search_begin(sl.plan, sl.series, 1, 0, 0);
    } else {
        rc = jerk_search_begin(sl.plan, pd.req.spectrum, pd.req.on_device, 0, 0);
    }
    if (rc != JERK_OK) {
        if (sl.series)
            cudaStreamSynchronize(s->stream);  // nothing may still read the buffer
        release_series(s, sl);
        release_bank(s, sl.key);
        s->idle.push_back(IdlePlan{sl.plan, sl.geo.obs, sl.key, sl.bytes});
        finish(s, pd.req, pd.t_submit, sl.t_start, rc, nullptr, 0);
        return true;
    }
    s->active.push_back(std::move(sl));
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->peak_bytes = std::max(s->peak_bytes, s->bytes_in_use);
    }
    return true;
}

static void worker_main(jerk_server *s)
{
    cudaSetDevice(s->cfg.device);
    for (;;) {
        // admission (requests queued before t_round all get a chance now)
        const double t_round = now_s();
        for (;;) {
            Pending pd;
            {
                std::unique_lock<std::mutex> lk(s->mu);
                if (s->stop && s->pending.empty() && s->active.empty())
                    goto out;
                if (s->pending.empty() || (int)s->active.size() >= s->cfg.max_active)
                    break;
                pd = s->pending.front();
            }
            if (!admit(s, pd))
                break;
            std::lock_guard<std::mutex> lk(s->mu);
            s->pending.pop_front();
        }
        // requests that had their admission chance this round and are still
        // waiting, longer than allowed, fail (later arrivals get theirs first)
        if (s->cfg.queue_timeout_s > 0) {
            std::vector<Pending> expired;
            {
                std::lock_guard<std::mutex> lk(s->mu);
                const double t = now_s();
                for (auto it = s->pending.begin(); it != s->pending.end();) {
                    if (it->t_submit < t_round && t - it->t_submit > s->cfg.queue_timeout_s) {
                        expired.push_back(*it);
                        it = s->pending.erase(it);
                    } else {
                        ++it;
                    }
                }
            }
            for (auto &pd : expired)
                finish(s, pd.req, pd.t_submit, now_s(), JERK_TIMEOUT, nullptr, 0);
        }
        // keep every active search a few batches ahead of the device, in
        // waves of merged launches over all of them
        bool progressed = false;
        {
            std::vector<jerk_plan *> plans;
            for (auto &sl : s->active)
                plans.push_back(sl.plan);
            if (!plans.empty())
                jerk_group_advance(plans.data(), (int)plans.size(),
                                   s->cfg.batches_ahead);  // errors: jerk_search_ready
        }

        // completions
        for (size_t i = 0; i < s->active.size();) {
            Slot &sl = s->active[i];
            const int ready = jerk_search_ready(sl.plan);
            if (ready == 0) {
                i++;
                continue;
            }
            jerk_cand *c = nullptr;
            long long n = 0;
            const int rc = ready < 0 ? ready : jerk_search_collect(sl.plan, &c, &n, nullptr);
            {
                // the plan's own copies: a host spectrum in, hit lists out
                long long h = 0, d = 0;
                jerk_plan_transfer_stats(sl.plan, &h, &d);
                jerk_plan_reset_stats(sl.plan);
                std::lock_guard<std::mutex> lk(s->mu);
                s->h2d_bytes += h;
                s->d2h_bytes += d;
            }
            release_bank(s, sl.key);
            if (sl.series) {
                if (rc < 0)
                    cudaStreamSynchronize(s->stream);  // a failed search may have left work queued
                release_series(s, sl);
            }
            if (rc < 0) {
                // a plan whose search failed is not reused
                jerk_plan_destroy(sl.plan);
                s->bytes_in_use -= sl.bytes;
            } else {
                s->idle.push_back(IdlePlan{sl.plan, sl.geo.obs, sl.key, sl.bytes});
            }
            finish(s, sl.req, sl.t_submit, sl.t_start, rc, c, n);
            s->active.erase(s->active.begin() + i);
            progressed = true;
        }
        if (!progressed) {
            std::unique_lock<std::mutex> lk(s->mu);
            const bool can_admit = !s->pending.empty() && (int)s->active.size() < s->cfg.max_active;
            if (!can_admit && !s->stop)
                s->cv_work.wait_for(lk, std::chrono::microseconds(s->active.empty() ? 20000 : 200));
        }
    }
out:
    for (auto &b : s->series_pool)
        jerk_device_free(b.ptr);
    s->series_pool.clear();
    for (auto &ip : s->idle)
        jerk_plan_destroy(ip.plan);
    s->idle.clear();
    for (auto &kv : s->banks)
        jerk_device_free(kv.second.ptr);
    s->banks.clear();
}

extern "C" int jerk_server_create(jerk_server **out, const jerk_server_config *cfg)
{
    if (!out)
        return JERK_EINVAL;
    jerk_server *s = new jerk_server();
    if (cfg)
        s->cfg = *cfg;
    if (s->cfg.max_active <= 0)
        s->cfg.max_active = 3;
    if (s->cfg.batch_rsteps <= 0)
        s->cfg.batch_rsteps = 16;
    if (s->cfg.batches_ahead <= 0)
        s->cfg.batches_ahead = 3;
    if (s->cfg.hbm_budget_bytes <= 0) {
        size_t fr = 0, tot = 0;
        cudaSetDevice(s->cfg.device);
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
            delete s;
            return JERK_ECUDA;
        }
        s->cfg.hbm_budget_bytes = (long long)(0.85 * (double)fr);
    }
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(s->cfg.device);
    const cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    cudaSetDevice(cur);
    if (e != cudaSuccess) {
        delete s;
        return JERK_ECUDA;
    }
    s->worker = std::thread(worker_main, s);
    *out = s;
    return JERK_OK;
}

extern "C" int jerk_server_submit(jerk_server *s, const jerk_request *req)
{
    if (!s || !req || !req->spectrum)
        return JERK_EINVAL;
    jerk_request r = *req;
    if (r.timeseries) {
        if (jerk_spectrum_scratch_bytes(r.N) <= 0)
            return JERK_EUNSUPPORTED;
        if (r.numbirds < 0 || (r.numbirds > 0 && (!r.bird_lobins || !r.bird_hibins)))
            return JERK_EINVAL;
        r.numbins = r.N / 2;
    } else {
        r.numbirds = 0;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop)
        return JERK_EINVAL;
    s->pending.push_back(Pending{r, now_s()});
    s->submitted++;
    s->cv_work.notify_all();
    return JERK_OK;
}

extern "C" int jerk_server_poll(jerk_server *s, jerk_result *out, int timeout_ms)
{
    if (!s || !out)
        return JERK_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms < 0 ? 0 : timeout_ms),
                             [&] { return !s->done.empty(); }))
        return JERK_TIMEOUT;
    *out = s->done.front();
    s->done.pop_front();
    return JERK_OK;
}

extern "C" void jerk_server_stats(jerk_server *s, long long *out)
{
    if (!s || !out)
        return;
    std::lock_guard<std::mutex> lk(s->mu);
    out[0] = s->submitted;
    out[1] = s->finished;
    out[2] = s->failed;
    out[3] = (long long)s->pending.size();
    out[4] = s->peak_bytes;
    out[5] = s->cfg.hbm_budget_bytes;
}

extern "C" void jerk_server_transfer_stats(jerk_server *s, long long *h2d, long long *d2h)
{
    long long h = 0, d = 0;
    if (s) {
        std::lock_guard<std::mutex> lk(s->mu);
        h = s->h2d_bytes;
        d = s->d2h_bytes;
    }
    if (h2d)
        *h2d = h;
    if (d2h)
        *d2h = d;
}

extern "C" void jerk_server_destroy(jerk_server *s)
{
    if (!s)
        return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv_work.notify_all();
    }
    if (s->worker.joinable())
        s->worker.join();
    for (auto &r : s->done)
        jerk_free(r.cands);
    if (s->stream)
        cudaStreamDestroy(s->stream);
    delete s;
}
