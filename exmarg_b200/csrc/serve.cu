// The native request loop: exm_serve_start / exm_serve_add_bank / exm_submit / exm_poll / exm_serve_stats /
// exm_serve_stop.  The reference analyses segments one pe_intrinsic call at a time (exmarg/search/pe.py:289-346);
// this loop keeps that call's results and adds continuous batching for callers in any language:
//
// * a request is one segment (H1, L1 data and noise, complex128 / float64 on the host, copied at submit) to
//   analyse with one of the server's banks and a random-draw seed;
// * a worker is a child context (exm_ctx_create_sharing: the parent's resident tables, its own stream, bank
//   and workspace) with a host thread of its own, so requests of different banks and segments run on the
//   device at the same time;
// * admission runs whenever a request arrives or a worker finishes: the oldest queued request that has an
//   idle worker of its bank starts on it; else, if its bank has no worker at all, idle workers of banks with
//   no queued request are closed until a new worker fits the HBM budget and the worker limit; a bank whose
//   workers are all busy gets another only from free budget (opening a worker -- context, workspace, FFT
//   plans, graph capture -- costs more than a segment).  Only a worker idle for at least the server's
//   minimum idle time (0.25 s by default) may be closed, so a mix of banks wider than the budget does not
//   close and reopen workers on every bank change; a dispatcher thread re-runs admission every 20 ms while
//   requests wait.  A worker's cost is first estimated from its bank's shape and replaced by the bytes its
//   context holds after its first segment;
// * a request that starts while r others run gets the r-th highest stream priority, so the oldest
//   segment's gather leads and the others fill its gaps;
// * every worker takes the parent's gather launch shape, so a result is bitwise the result of
//   exm_pe_intrinsic on the parent for the same bank, segment and seed, whatever else is running.
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>

#include "common.cuh"
#include "kernels.cuh"

namespace {

struct SrvBank {
    int nm = 0, nfreq = 0, lo = 0, nt = 0;
    std::vector<float> W;
    std::vector<double> u, M, q, chi, lny, p;
    double ymin = 0.0;
    int prior = EXM_PRIOR_VOLUME;
    size_t cost = 0;
    bool measured = false;
};

struct SrvRequest {
    int64_t id = 0;
    int bank = 0;
    int64_t seed = 0;
    std::vector<double> dH, dL, s2H, s2L;
    bool done = false;
    int rc = EXM_OK;
    std::string msg;
    std::vector<double> lnl;
    double lnb = 0.0;
};

struct SrvWorker {
    int id = 0, bank = 0;
    exm_ctx *ctx = nullptr;
    std::thread th;
    std::condition_variable cv;
    std::shared_ptr<SrvRequest> job;
    int rank = 0;           // requests already on the device when the job was assigned
    double t_idle = 0.0;    // when the worker last became idle
    bool stop = false;
    bool waiting = false;   // parked on cv: the only state in which another thread may close it
};

double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

struct exm_server {
    exm_ctx *parent = nullptr;
    size_t budget = 0, used = 0;
    int max_workers = 1, n_loud = 0, n_random = 0, graph = 0;
    std::mutex mu;
    std::condition_variable cv_done;
    std::vector<SrvBank> banks;
    std::deque<std::shared_ptr<SrvRequest>> queue;
    std::map<int64_t, std::shared_ptr<SrvRequest>> reqs;
    std::map<int, std::unique_ptr<SrvWorker>> workers;
    int64_t next_req = 1;
    int next_worker = 0, n_running = 0;
    long long n_served = 0, n_failed = 0, n_created = 0, n_evicted = 0;
    double t_first = 0.0, t_last = 0.0;
    double min_idle_s = 0.25;          // an idle worker is closed for another bank only after this long
    bool stopping = false;
    std::condition_variable cv_disp;   // wakes the dispatcher when requests are queued
    std::thread dispatcher;
};

// device bytes one worker's workspace takes for a bank (as exm_pe_intrinsic sizes it): the FFT rows and
// trajectories, selection, tap descriptors, partial sums and the bank, plus cuFFT's work area
static size_t workspace_estimate(const exm_server *s, const SrvBank &b)
{
    const exm_ctx *p = s->parent;
    const size_t nm = b.nm, nt = b.nt, nmc = std::min<size_t>(nm, EXM_MAX_CHUNK);
    const size_t nwalk = s->n_loud > 0 ? (size_t)(s->n_loud + s->n_random) : nt;
    const size_t per_lag = nmc * nwalk * 20;
    const size_t rc = std::max<size_t>(1, std::min<size_t>((size_t)p->ntau, ((size_t)8 << 30) / std::max<size_t>(per_lag, 1)));
    size_t by = 2 * nmc * nt * (16 + 8 + 4);   // FFT rows, trajectories, ln|z| residuals
    by += std::max(nmc * nt, nm * 1024 + 4096) * 4 + nm * 1024 * 4;
    by += nmc * nwalk * 4 + rc * 48 * (nmc + 1) * 4 + rc * per_lag;
    by += (size_t)(p->nn + 1) * p->ntau * nm * 8 + nm * 8 * 12 + nm * (size_t)b.nfreq * 8;
    by += 2 * nm * nt * 16 / std::max<size_t>(1, nm / std::max<size_t>(nmc, 1));
    return (size_t)((double)by * 1.05) + ((size_t)64 << 20);
}

static void worker_main(exm_server *s, SrvWorker *w);

// one worker of bank b, started on its own thread (which opens its context); mu held
static SrvWorker *open_worker(exm_server *s, int b)
{
    std::unique_ptr<SrvWorker> w(new SrvWorker());
    w->id = s->next_worker++;
    w->bank = b;
    SrvWorker *raw = w.get();
    s->workers[w->id] = std::move(w);
    s->used += s->banks[b].cost;
    s->n_created += 1;
    raw->th = std::thread(worker_main, s, raw);
    return raw;
}

// an idle worker of a bank other than `need` that has no queued request, detached from the server (mu held)
static std::unique_ptr<SrvWorker> evict_one(exm_server *s, int need)
{
    std::vector<char> waiting(s->banks.size(), 0);
    for (auto &r : s->queue) waiting[r->bank] = 1;
    for (auto it = s->workers.begin(); it != s->workers.end(); ++it) {
        SrvWorker *w = it->second.get();
        if (w->bank == need || waiting[w->bank] || w->job || !w->waiting) continue;
        if (now_s() - w->t_idle < s->min_idle_s) continue;   // recently used: keep it
        std::unique_ptr<SrvWorker> out = std::move(it->second);
        s->workers.erase(it);
        s->used -= std::min(s->used, s->banks[out->bank].cost);
        s->n_evicted += 1;
        return out;
    }
    return nullptr;
}

// admit every queued request that can start now (mu held); workers closed for budget are returned for the
// caller to join after releasing mu
static void admit(exm_server *s, std::vector<std::unique_ptr<SrvWorker>> &closed)
{
    bool progress = true;
    while (progress && !s->stopping) {
        progress = false;
        for (auto qi = s->queue.begin(); qi != s->queue.end(); ++qi) {
            const int b = (*qi)->bank;
            SrvWorker *w = nullptr;
            int mine = 0;
            for (auto &kv : s->workers)
                if (kv.second->bank == b) {
                    ++mine;
                    if (!w && !kv.second->job) w = kv.second.get();
                }
            if (!w) {
                const size_t c = s->banks[b].cost;
                while (mine == 0 && (s->used + c > s->budget || (int)s->workers.size() >= s->max_workers)) {
                    std::unique_ptr<SrvWorker> e = evict_one(s, b);
                    if (!e) break;
                    e->stop = true;
                    e->cv.notify_all();
                    closed.push_back(std::move(e));
                }
                if ((int)s->workers.size() < s->max_workers && s->used + c <= s->budget) w = open_worker(s, b);
            }
            if (w) {
                w->job = *qi;
                w->rank = s->n_running++;
                s->queue.erase(qi);
                w->cv.notify_all();
                progress = true;
                break;
            }
        }
    }
}

static void join_closed(std::vector<std::unique_ptr<SrvWorker>> &closed)
{
    for (auto &w : closed)
        if (w->th.joinable()) w->th.join();
    closed.clear();
}

static void finish(exm_server *s, SrvRequest &r, int rc, const std::string &msg)
{
    r.rc = rc;
    r.msg = msg;
    r.done = true;
    if (rc == EXM_OK) s->n_served += 1; else s->n_failed += 1;
    s->t_last = now_s();
}

static void worker_main(exm_server *s, SrvWorker *w)
{
    const SrvBank &bk = s->banks[w->bank];   // banks are only appended before the first submit
    int rc = exm_ctx_create_sharing(s->parent, 0, &w->ctx);
    std::string err = rc == EXM_OK ? "" : "opening a worker context failed";
    if (rc == EXM_OK) {
        rc = exm_bank_set(w->ctx, bk.nm, bk.nfreq, bk.lo, bk.nt, bk.W.data(), bk.u.data(), bk.M.data(), bk.q.data(),
                          bk.chi.data());
        if (rc == EXM_OK)
            rc = exm_pe_prepare(w->ctx, bk.ymin, bk.prior, bk.lny.empty() ? nullptr : bk.lny.data(),
                                bk.p.empty() ? nullptr : bk.p.data(), (int)bk.lny.size());
        if (rc == EXM_OK && s->graph) rc = exm_ctx_set_graph(w->ctx, 1);
        if (rc != EXM_OK) err = std::string(w->ctx->err);
    }
    int greatest = 0, least = 0;
    cudaSetDevice(s->parent->dev);
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess) least = greatest = 0;
    int prio = 0;
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        w->waiting = true;
        w->cv.wait(lk, [&] { return w->stop || w->job; });
        w->waiting = false;
        if (!w->job) break;   // stopped while idle
        std::shared_ptr<SrvRequest> r = w->job;
        const int rank = w->rank;
        lk.unlock();
        int rc2 = rc;
        std::string msg = err;
        std::vector<double> lnl(bk.nm);
        double lnb = 0.0;
        size_t bytes = 0;
        if (rc2 == EXM_OK) {
            const int want = std::min(least, greatest + rank);
            if (want != prio && exm_ctx_set_priority(w->ctx, want, nullptr) == EXM_OK) prio = want;
            rc2 = exm_pe_intrinsic(w->ctx, 1, r->dH.data(), r->dL.data(), r->s2H.data(), r->s2L.data(), &r->seed,
                                   s->n_loud, s->n_random, lnl.data(), &lnb);
            if (rc2 != EXM_OK) msg = std::string(w->ctx->err);
            bytes = w->ctx->used;
        }
        std::vector<std::unique_ptr<SrvWorker>> closed;
        lk.lock();
        s->n_running -= 1;
        r->lnl.swap(lnl);
        r->lnb = lnb;
        finish(s, *r, rc2, msg);
        w->job.reset();
        w->t_idle = now_s();
        SrvBank &b = s->banks[w->bank];
        if (rc2 == EXM_OK && !b.measured) {   // the estimate gives way to the measured size
            size_t n_of_bank = 0;
            for (auto &kv : s->workers) n_of_bank += kv.second->bank == w->bank;
            s->used = s->used - std::min(s->used, b.cost * n_of_bank) + bytes * n_of_bank;
            b.cost = bytes;
            b.measured = true;
        }
        s->cv_done.notify_all();
        if (rc != EXM_OK) {   // a worker that could not open serves nothing more: close it
            auto it = s->workers.find(w->id);
            if (it != s->workers.end()) {
                it->second->th.detach();
                s->used -= std::min(s->used, b.cost);
                std::unique_ptr<SrvWorker> self = std::move(it->second);
                s->workers.erase(it);
                admit(s, closed);
                lk.unlock();
                join_closed(closed);
                if (w->ctx) exm_ctx_destroy(w->ctx);
                return;   // `self` frees this worker's record
            }
        }
        admit(s, closed);
        if (!closed.empty()) {
            lk.unlock();
            join_closed(closed);
            lk.lock();
        }
    }
    lk.unlock();
    if (w->ctx) exm_ctx_destroy(w->ctx);
    w->ctx = nullptr;
}

// re-runs admission while requests are queued (a closing rule may hold them until a worker has idled long
// enough, with no submit or finish to trigger admission again)
static void dispatcher_main(exm_server *s)
{
    std::unique_lock<std::mutex> lk(s->mu);
    while (!s->stopping) {
        s->cv_disp.wait_for(lk, std::chrono::milliseconds(20), [&] { return s->stopping; });
        if (s->stopping || s->queue.empty()) continue;
        std::vector<std::unique_ptr<SrvWorker>> closed;
        admit(s, closed);
        if (!closed.empty()) {
            lk.unlock();
            join_closed(closed);
            lk.lock();
        }
    }
}

#define SRV_BEGIN(ctx)                                                                                             \
    if (!(ctx)) return EXM_ERR_ARG;                                                                                \
    try {
#define SRV_END(ctx)                                                                                               \
    }                                                                                                              \
    catch (const exm_error &e)                                                                                     \
    {                                                                                                              \
        (ctx)->err = e.msg;                                                                                        \
        return e.code;                                                                                             \
    }                                                                                                              \
    catch (const std::exception &e)                                                                                \
    {                                                                                                              \
        (ctx)->err = e.what();                                                                                     \
        return EXM_ERR_OOM;                                                                                        \
    }                                                                                                              \
    return EXM_OK;

extern "C" int exm_serve_start(exm_ctx *ctx, size_t hbm_budget, int max_workers, int n_loud, int n_random,
                               int use_graph)
{
    SRV_BEGIN(ctx)
    if (ctx->srv) EXM_THROW(EXM_ERR_STATE, "a server is already running on this context");
    if (ctx->store_borrowed) EXM_THROW(EXM_ERR_STATE, "serve from the context that owns the store");
    if (!ctx->store_ok) EXM_THROW(EXM_ERR_STATE, "store is not complete (exm_store_init + every node)");
    if (ctx->shard) EXM_THROW(EXM_ERR_STATE, "a store shard cannot serve ln Lambda");
    if (max_workers < 1 || max_workers > 64) EXM_THROW(EXM_ERR_ARG, "max_workers must be 1..64");
    if (n_loud < 0 || n_random < 0 || (n_loud > 0 && n_random < 1))
        EXM_THROW(EXM_ERR_ARG, "n_loud >= 0, and n_random >= 1 when n_loud > 0");
    EXM_CUDA(cudaSetDevice(ctx->dev));
    std::unique_ptr<exm_server> s(new exm_server());
    s->parent = ctx;
    if (!hbm_budget) {
        size_t fr = 0, tot = 0;
        EXM_CUDA(cudaMemGetInfo(&fr, &tot));
        hbm_budget = (size_t)(0.85 * (double)fr);
    }
    s->budget = hbm_budget;
    s->max_workers = max_workers;
    s->n_loud = n_loud;
    s->n_random = n_random;
    s->graph = use_graph ? 1 : 0;
    s->dispatcher = std::thread(dispatcher_main, s.get());
    ctx->srv = s.release();
    SRV_END(ctx)
}

extern "C" int exm_serve_add_bank(exm_ctx *ctx, int nm, int nfreq, int lo, int n_time, const float *W,
                                  const double *u, const double *M, const double *q, const double *chi, double ymin,
                                  int prior, const double *lny, const double *p_lny, int n_dens, int *bank_id)
{
    SRV_BEGIN(ctx)
    exm_server *s = ctx->srv;
    if (!s) EXM_THROW(EXM_ERR_STATE, "no server on this context (exm_serve_start)");
    if (!bank_id || !W || !u || !M || !q || !chi) EXM_THROW(EXM_ERR_ARG, "null bank argument");
    if (nm < 1 || nm > EXM_MAX_CHUNK || nfreq < 1 || lo < 0 || lo + nfreq > n_time)
        EXM_THROW(EXM_ERR_ARG, "a served bank needs 1..8192 templates and lo + nfreq <= n_time");
    if (prior == EXM_PRIOR_TABULATED && (!lny || !p_lny || n_dens < 2))
        EXM_THROW(EXM_ERR_ARG, "a tabulated prior needs its density");
    if (prior != EXM_PRIOR_VOLUME && prior != EXM_PRIOR_TABULATED) EXM_THROW(EXM_ERR_ARG, "unknown prior");
    std::lock_guard<std::mutex> lk(s->mu);
    if (!s->reqs.empty() || s->n_served || s->n_failed)
        EXM_THROW(EXM_ERR_STATE, "add every bank before the first request");
    SrvBank b;
    b.nm = nm;
    b.nfreq = nfreq;
    b.lo = lo;
    b.nt = n_time;
    b.W.assign(W, W + (size_t)2 * nm * nfreq);
    b.u.assign(u, u + nm);
    b.M.assign(M, M + nm);
    b.q.assign(q, q + nm);
    b.chi.assign(chi, chi + nm);
    b.ymin = ymin;
    b.prior = prior;
    if (prior == EXM_PRIOR_TABULATED) {
        b.lny.assign(lny, lny + n_dens);
        b.p.assign(p_lny, p_lny + n_dens);
    }
    b.cost = workspace_estimate(s, b);
    s->banks.push_back(std::move(b));
    *bank_id = (int)s->banks.size() - 1;
    SRV_END(ctx)
}

extern "C" int exm_submit(exm_ctx *ctx, int bank_id, const double *d_H, const double *d_L, const double *sig2_H,
                          const double *sig2_L, int64_t seed, int64_t *handle)
{
    SRV_BEGIN(ctx)
    exm_server *s = ctx->srv;
    if (!s) EXM_THROW(EXM_ERR_STATE, "no server on this context (exm_serve_start)");
    if (!handle || !d_H || !d_L || !sig2_H || !sig2_L) EXM_THROW(EXM_ERR_ARG, "null request argument");
    if (seed < 0) EXM_THROW(EXM_ERR_ARG, "seed must be non-negative");
    std::shared_ptr<SrvRequest> r(new SrvRequest());
    std::vector<std::unique_ptr<SrvWorker>> closed;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stopping) EXM_THROW(EXM_ERR_STATE, "the server is stopping");
        if (bank_id < 0 || bank_id >= (int)s->banks.size()) EXM_THROW(EXM_ERR_ARG, "unknown bank id");
        const size_t nf = s->banks[bank_id].nfreq;
        r->bank = bank_id;
        r->seed = seed;
        r->dH.assign(d_H, d_H + 2 * nf);
        r->dL.assign(d_L, d_L + 2 * nf);
        r->s2H.assign(sig2_H, sig2_H + nf);
        r->s2L.assign(sig2_L, sig2_L + nf);
        r->id = s->next_req++;
        if (s->reqs.empty() && s->queue.empty() && s->n_running == 0) s->t_first = now_s();
        s->reqs[r->id] = r;
        s->queue.push_back(r);
        *handle = r->id;
        admit(s, closed);
    }
    join_closed(closed);
    SRV_END(ctx)
}

extern "C" int exm_poll(exm_ctx *ctx, int64_t handle, int64_t timeout_us, double *ln_lambda, double *ln_b)
{
    SRV_BEGIN(ctx)
    exm_server *s = ctx->srv;
    if (!s) EXM_THROW(EXM_ERR_STATE, "no server on this context (exm_serve_start)");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(handle);
    if (it == s->reqs.end()) EXM_THROW(EXM_ERR_ARG, "unknown request handle (never submitted, or already polled)");
    std::shared_ptr<SrvRequest> r = it->second;
    if (timeout_us < 0)
        s->cv_done.wait(lk, [&] { return r->done; });
    else if (timeout_us > 0)
        s->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us), [&] { return r->done; });
    if (!r->done) {
        ctx->err = "request " + std::to_string(handle) + " has not finished";
        return EXM_ERR_TIMEOUT;
    }
    s->reqs.erase(it);
    if (r->rc != EXM_OK) {
        ctx->err = r->msg;
        return r->rc;
    }
    if (ln_lambda) std::copy(r->lnl.begin(), r->lnl.end(), ln_lambda);
    if (ln_b) *ln_b = r->lnb;
    SRV_END(ctx)
}

extern "C" int exm_serve_stats(exm_ctx *ctx, double *out)
{
    SRV_BEGIN(ctx)
    exm_server *s = ctx->srv;
    if (!s) EXM_THROW(EXM_ERR_STATE, "no server on this context (exm_serve_start)");
    if (!out) EXM_THROW(EXM_ERR_ARG, "null output");
    std::lock_guard<std::mutex> lk(s->mu);
    out[0] = (double)s->n_served;
    out[1] = (double)s->n_failed;
    out[2] = (double)s->queue.size();
    out[3] = (double)s->n_running;
    out[4] = (double)s->workers.size();
    out[5] = (double)s->n_created;
    out[6] = (double)s->n_evicted;
    out[7] = (double)s->used;
    out[8] = (double)s->budget;
    out[9] = s->t_last > s->t_first ? s->t_last - s->t_first : 0.0;
    SRV_END(ctx)
}

// Stop the server of ctx: running requests finish, queued ones fail with EXM_ERR_STATE (their handles stay
// pollable until the server is gone: poll before stopping), every worker is closed.  Called by
// exm_ctx_destroy for a context that still serves.
void exm_serve_destroy(exm_ctx *ctx)
{
    exm_server *s = ctx->srv;
    if (!s) return;
    std::vector<std::unique_ptr<SrvWorker>> all;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        s->stopping = true;
        s->cv_disp.notify_all();
        for (auto &r : s->queue) finish(s, *r, EXM_ERR_STATE, "the server stopped before the request started");
        s->queue.clear();
        s->cv_done.wait(lk, [&] { return s->n_running == 0; });
        for (auto &kv : s->workers) {
            kv.second->stop = true;
            kv.second->cv.notify_all();
            all.push_back(std::move(kv.second));
        }
        s->workers.clear();
        s->cv_done.notify_all();
    }
    if (s->dispatcher.joinable()) s->dispatcher.join();
    join_closed(all);
    ctx->srv = nullptr;
    delete s;
}

extern "C" int exm_serve_set_min_idle(exm_ctx *ctx, double seconds)
{
    SRV_BEGIN(ctx)
    exm_server *s = ctx->srv;
    if (!s) EXM_THROW(EXM_ERR_STATE, "no server on this context (exm_serve_start)");
    if (!(seconds >= 0.0 && seconds <= 3600.0)) EXM_THROW(EXM_ERR_ARG, "minimum idle time must be 0..3600 s");
    std::lock_guard<std::mutex> lk(s->mu);
    s->min_idle_s = seconds;
    SRV_END(ctx)
}

extern "C" int exm_serve_stop(exm_ctx *ctx)
{
    SRV_BEGIN(ctx)
    if (!ctx->srv) EXM_THROW(EXM_ERR_STATE, "no server on this context");
    exm_serve_destroy(ctx);
    SRV_END(ctx)
}
