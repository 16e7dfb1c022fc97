// The C ABI (include/exmarg_b200.h): context, store, bank, the prepared geometry and
// the pe_intrinsic pipeline (filter -> select_times -> taps -> plane gather ->
// node / distance log-sum-exp -> ln B), plus the stage entry points.
#include <cmath>
#include <cstring>
#include <new>
#include <numeric>

#include <mutex>

#include <nvtx3/nvToolsExt.h>

#include "common.cuh"
#include "kernels.cuh"
#include "pcg64.cuh"

void exm_make_tmap(exm_ctx *ctx);
void exm_store_generate(exm_ctx *ctx, int k, const float *M, const float *P, const float *Q, float S, uint32_t seed);
void exm_run_node_values(exm_ctx *ctx, exm_slot &sl, double *d_lamN);
void exm_run_distance_weights_y(exm_ctx *ctx, const double *d_y, double ymin, int prior, const double *d_lny,
                                const double *d_p, int n_dens, const double *d_gl);
void exm_run_topk(exm_ctx *ctx, exm_slot &sl, int nmc, const int *d_order_chunk, int K, int S);
void exm_run_np_exp32(exm_ctx *ctx, const float *d_x, float *d_y, long long n);
void exm_noalloc_load(int dev);
void exm_serve_destroy(exm_ctx *ctx);

// ------------------------------------------------------------------ memory

void exm_alloc(exm_ctx *ctx, dbuf &b, size_t bytes)
{
    if (bytes == 0) bytes = 256;
    if (ctx->used + bytes > ctx->budget)
        EXM_THROW(EXM_ERR_OOM, "device memory budget exceeded: need " + std::to_string(bytes) + " more bytes, " +
                                   std::to_string(ctx->budget - ctx->used) + " left of " +
                                   std::to_string(ctx->budget));
    void *p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        EXM_THROW(EXM_ERR_OOM, std::string("cudaMalloc of ") + std::to_string(bytes) + " bytes: " + cudaGetErrorString(e));
    }
    b.p = p;
    b.bytes = bytes;
    ctx->used += bytes;
    ctx->alloc_gen++;
}

void exm_free(exm_ctx *ctx, dbuf &b)
{
    if (b.p) {
        cudaFree(b.p);
        ctx->used -= b.bytes;
        ctx->alloc_gen++;
    }
    b.p = nullptr;
    b.bytes = 0;
}

void exm_ensure(exm_ctx *ctx, dbuf &b, size_t bytes)
{
    if (b.p && b.bytes >= bytes) return;
    exm_free(ctx, b);
    exm_alloc(ctx, b, bytes);
}

static void free_slot(exm_ctx *ctx, exm_slot &s)
{
    dbuf *all[] = {&s.traj, &s.trajlo, &s.fft, &s.keys, &s.picks, &s.rej, &s.sel, &s.hist, &s.win, &s.cnt,
                   &s.desc, &s.tside, &s.part, &s.lnl, &s.lnb, &s.dev_err, &s.din};
    for (dbuf *b : all) exm_free(ctx, *b);
    if (s.hostin.p) cudaFreeHost(s.hostin.p);
    s.hostin.p = nullptr;
    s.hostin.bytes = 0;
}

void exm_fft_plan(exm_ctx *ctx, int batch)
{
    if (ctx->plan && ctx->plan_batch == batch && ctx->plan_n == ctx->nt) return;
    if (ctx->plan) cufftDestroy(ctx->plan);
    ctx->plan = 0;
    EXM_CUFFT(cufftCreate(&ctx->plan));
    EXM_CUFFT(cufftSetAutoAllocation(ctx->plan, 0));
    long long n = ctx->nt;
    size_t ws = 0;
    EXM_CUFFT(cufftMakePlanMany64(ctx->plan, 1, &n, nullptr, 1, n, nullptr, 1, n, CUFFT_Z2Z, batch, &ws));
    exm_ensure(ctx, ctx->fftwork, ws);
    EXM_CUFFT(cufftSetWorkArea(ctx->plan, ctx->fftwork.p));
    EXM_CUFFT(cufftSetStream(ctx->plan, ctx->stream));
    ctx->plan_batch = batch;
    ctx->plan_n = ctx->nt;
}

// ------------------------------------------------------------------ stage timers

int exm_tim_begin(exm_ctx *ctx, int stage)
{
    if (!ctx->tim_on) return -1;
    if (ctx->ev_used == ctx->ev_pool.size()) {
        std::pair<cudaEvent_t, cudaEvent_t> e;
        EXM_CUDA(cudaEventCreate(&e.first));
        EXM_CUDA(cudaEventCreate(&e.second));
        ctx->ev_pool.push_back(e);
    }
    const int h = (int)ctx->ev_used++;
    EXM_CUDA(cudaEventRecord(ctx->ev_pool[h].first, ctx->stream));
    ctx->ev_pending.push_back({stage, h});
    return h;
}

void exm_tim_end(exm_ctx *ctx, int h)
{
    if (h < 0) return;
    EXM_CUDA(cudaEventRecord(ctx->ev_pool[h].second, ctx->stream));
}

void exm_tim_collect(exm_ctx *ctx)
{
    for (auto &pe : ctx->ev_pending) {
        float ms = 0.f;
        EXM_CUDA(cudaEventElapsedTime(&ms, ctx->ev_pool[pe.second].first, ctx->ev_pool[pe.second].second));
        ctx->tacc[pe.first] += ms;
    }
    ctx->ev_pending.clear();
    ctx->ev_used = 0;
}

// ------------------------------------------------------------------ api plumbing

#define API_BEGIN(ctx)                                                                                             \
    if (!(ctx)) return EXM_ERR_ARG;                                                                                \
    try {
#define API_END(ctx)                                                                                               \
    }                                                                                                              \
    catch (const exm_error &e)                                                                                     \
    {                                                                                                              \
        (ctx)->err = e.msg;                                                                                        \
        return e.code;                                                                                             \
    }                                                                                                              \
    catch (const std::exception &e)                                                                                \
    {                                                                                                              \
        (ctx)->err = e.what();                                                                                     \
        return EXM_ERR_CUDA;                                                                                       \
    }                                                                                                              \
    return EXM_OK;

#define REQUIRE(cond, code, msg)                                                                                   \
    do {                                                                                                           \
        if (!(cond)) EXM_THROW(code, msg);                                                                         \
    } while (0)

extern "C" int exm_ctx_timing(exm_ctx *ctx, int enable, double *out)
{
    API_BEGIN(ctx)
    if (out) {
        unsigned long long st[4] = {0, 0, 0, 0};
        if (ctx->d_stats.p) {
            EXM_CUDA(cudaMemcpy(st, ctx->d_stats.p, sizeof(st), cudaMemcpyDeviceToHost));
            EXM_CUDA(cudaMemset(ctx->d_stats.p, 0, sizeof(st)));
        }
        out[11] = (double)st[0];
        out[12] = (double)st[1];
        for (int i = 0; i < 6; ++i) out[i] = ctx->tacc[i];
        out[6] = (double)ctx->gather_launches;
        out[7] = ctx->node_taps;
        out[8] = ctx->tlw;
        out[9] = ctx->segments;
        out[10] = (double)ctx->launches;
    }
    for (double &t : ctx->tacc) t = 0.0;
    ctx->node_taps = ctx->tlw = ctx->segments = 0;
    ctx->gather_launches = ctx->launches = 0;
    ctx->tim_on = enable != 0;
    API_END(ctx)
}

extern "C" int exm_version(void) { return 10000; }

extern "C" int exm_device_memory(int device, size_t *free_bytes, size_t *total_bytes)
{
    if (!free_bytes || !total_bytes) return EXM_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess || cudaMemGetInfo(free_bytes, total_bytes) != cudaSuccess) {
        (void)cudaGetLastError();
        return EXM_ERR_CUDA;
    }
    return EXM_OK;
}

extern "C" int exm_rng_integers(uint64_t seed, uint32_t high, int64_t count, int64_t *out)
{
    if (high < 1 || count < 0 || (count > 0 && !out)) return EXM_ERR_ARG;
    exm_pcg g = exm_pcg_from_seed(seed);
    const uint32_t rng = high - 1;
    if (rng == 0) {
        for (int64_t i = 0; i < count; ++i) out[i] = 0;
        return EXM_OK;
    }
    const uint32_t thr = (uint32_t)((1ull << 32) % high);
    uint64_t buf = 0;
    bool have = false;
    for (int64_t i = 0; i < count;) {
        uint32_t x;
        if (have) {
            x = (uint32_t)(buf >> 32);
            have = false;
        } else {
            exm_pcg_step(g);
            buf = exm_pcg_output(g.state);
            x = (uint32_t)buf;
            have = true;
        }
        const uint64_t m = (uint64_t)x * high;
        if ((uint32_t)m < thr) continue;
        out[i++] = (int64_t)(m >> 32);
    }
    return EXM_OK;
}

extern "C" int exm_ctx_create(int device, size_t hbm_budget, exm_ctx **out)
{
    if (!out) return EXM_ERR_ARG;
    *out = nullptr;
    exm_ctx *ctx = new (std::nothrow) exm_ctx();
    if (!ctx) return EXM_ERR_OOM;
    try {
        EXM_CUDA(cudaSetDevice(device));
        ctx->dev = device;
        EXM_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        cudaDeviceProp pr;
        EXM_CUDA(cudaGetDeviceProperties(&pr, device));
        ctx->sm_count = pr.multiProcessorCount;
        ctx->smem_optin = pr.sharedMemPerBlockOptin;
        if (pr.major < 10) EXM_THROW(EXM_ERR_CUDA, "libexmarg_b200 is built for sm_100a (B200); device is sm_" +
                                                       std::to_string(pr.major * 10 + pr.minor));
        size_t fr = 0, tot = 0;
        EXM_CUDA(cudaMemGetInfo(&fr, &tot));
        ctx->budget = hbm_budget ? hbm_budget : (size_t)(0.9 * (double)fr);
        exm_noalloc_load(device);   // exm_gather_noalloc's fixed scratch and kernels, loaded now
    } catch (const exm_error &e) {
        fprintf(stderr, "exm_ctx_create: %s\n", e.msg.c_str());
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        delete ctx;
        return e.code;
    } catch (const std::exception &e) {
        fprintf(stderr, "exm_ctx_create: %s\n", e.what());
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        delete ctx;
        return EXM_ERR_OOM;
    }
    *out = ctx;
    return EXM_OK;
}

extern "C" int exm_ctx_create_sharing(exm_ctx *parent, size_t hbm_budget, exm_ctx **out)
{
    if (!parent || !out) return EXM_ERR_ARG;
    *out = nullptr;
    if (parent->store_borrowed) parent = parent->parent;   // share the owner's store, not a child's
    if (!parent->store_ok) {
        parent->err = "the parent context has no complete store to share";
        return EXM_ERR_STATE;
    }
    exm_ctx *ctx = new (std::nothrow) exm_ctx();
    if (!ctx) {
        parent->err = "host memory exhausted";
        return EXM_ERR_OOM;
    }
    try {
        EXM_CUDA(cudaSetDevice(parent->dev));
        ctx->dev = parent->dev;
        EXM_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        ctx->sm_count = parent->sm_count;
        ctx->smem_optin = parent->smem_optin;
        size_t fr = 0, tot = 0;
        EXM_CUDA(cudaMemGetInfo(&fr, &tot));
        ctx->budget = hbm_budget ? hbm_budget : (size_t)(0.9 * (double)fr);
        ctx->store_ok = true;
        ctx->store_borrowed = true;
        ctx->nn = parent->nn;
        ctx->ntau = parent->ntau;
        ctx->nphif = parent->nphif;
        ctx->nb = parent->nb;
        ctx->nd = parent->nd;
        ctx->ndp = parent->ndp;
        ctx->dtype = parent->dtype;
        ctx->beta0 = parent->beta0;
        ctx->dbeta = parent->dbeta;
        ctx->delta0 = parent->delta0;
        ctx->ddelta = parent->ddelta;
        ctx->tau = parent->tau;
        ctx->s = parent->s;
        ctx->alo = parent->alo;
        ctx->ahi = parent->ahi;
        ctx->node_set = parent->node_set;
        ctx->shard = parent->shard;
        ctx->s_before = parent->s_before;
        ctx->T.p = parent->T.p;            // borrowed: not counted, not freed
        ctx->tscale = parent->tscale;
        ctx->d_tscale.p = parent->d_tscale.p;
        ctx->tstride = parent->tstride;
        ctx->d_tau.p = parent->d_tau.p;
        ctx->tmap = parent->tmap;
        ctx->tmap_ok = parent->tmap_ok;
        ctx->gather_cfg = parent->gather_cfg;
        ctx->gather_chunk_pct = parent->gather_chunk_pct;
        ctx->traj_fp64 = parent->traj_fp64;
        exm_ensure(ctx, ctx->d_stats, 4 * sizeof(unsigned long long));
        EXM_CUDA(cudaMemset(ctx->d_stats.p, 0, 4 * sizeof(unsigned long long)));
    } catch (const exm_error &e) {
        parent->err = e.msg;
        exm_free(ctx, ctx->d_stats);
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        delete ctx;
        return e.code;
    } catch (const std::exception &e) {
        parent->err = e.what();
        exm_free(ctx, ctx->d_stats);
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        delete ctx;
        return EXM_ERR_OOM;
    }
    ctx->parent = parent;
    parent->n_children.fetch_add(1);
    *out = ctx;
    return EXM_OK;
}

extern "C" int exm_ctx_set_priority(exm_ctx *ctx, int priority, int *range_out)
{
    API_BEGIN(ctx)
    EXM_CUDA(cudaSetDevice(ctx->dev));
    int least = 0, greatest = 0;
    EXM_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    if (range_out) {
        range_out[0] = greatest;
        range_out[1] = least;
    }
    const int prio = std::min(least, std::max(greatest, priority));
    cudaStream_t s = nullptr;
    EXM_CUDA(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, prio));
    EXM_CUDA(cudaStreamSynchronize(ctx->stream));
    cudaStreamDestroy(ctx->stream);
    ctx->stream = s;
    if (ctx->plan) EXM_CUFFT(cufftSetStream(ctx->plan, ctx->stream));
    API_END(ctx)
}

extern "C" int exm_ctx_set_graph(exm_ctx *ctx, int enable)
{
    if (!ctx) return EXM_ERR_ARG;
    ctx->use_graph = enable != 0;
    return EXM_OK;
}

static void ctx_free(exm_ctx *ctx)
{
    cudaSetDevice(ctx->dev);
    cudaStreamSynchronize(ctx->stream);
    exm_redshift_release(ctx);
    if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
    if (ctx->plan) cufftDestroy(ctx->plan);
    if (ctx->store_borrowed) {   // the parent owns the tables
        ctx->T = dbuf();
        ctx->d_tau = dbuf();
        ctx->d_tscale = dbuf();
    }
    free_slot(ctx, ctx->slot);
    for (auto &e : ctx->ev_pool) {
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    dbuf *all[] = {&ctx->T, &ctx->d_tau, &ctx->d_tscale, &ctx->d_W, &ctx->d_bhat_off, &ctx->d_bnode, &ctx->d_cb, &ctx->d_lnW,
                   &ctx->d_cell, &ctx->d_mlo, &ctx->d_mhi, &ctx->d_order, &ctx->d_cki, &ctx->d_ckd, &ctx->fftwork, &ctx->d_stats};
    for (dbuf *b : all) exm_free(ctx, *b);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
}

static std::mutex g_attr_mu;
struct AttrDone {
    int dev;
    const void *func;
    size_t max_dyn;   // the dynamic shared memory the function may take on this device
};
static std::vector<AttrDone> g_attr_done;

void exm_allow_smem(exm_ctx *ctx, const void *func, size_t smem)
{
    std::lock_guard<std::mutex> lock(g_attr_mu);
    size_t max_dyn = 0;
    bool found = false;
    for (const AttrDone &d : g_attr_done)
        if (d.dev == ctx->dev && d.func == func) {
            max_dyn = d.max_dyn;
            found = true;
        }
    if (!found) {
        cudaFuncAttributes fa;
        EXM_CUDA(cudaFuncGetAttributes(&fa, func));
        // the opt-in limit covers static and dynamic shared memory together
        max_dyn = ctx->smem_optin > fa.sharedSizeBytes ? ctx->smem_optin - fa.sharedSizeBytes : 0;
        EXM_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)max_dyn));
        g_attr_done.push_back({ctx->dev, func, max_dyn});
    }
    if (smem > max_dyn)
        EXM_THROW(EXM_ERR_ARG, "a kernel needs " + std::to_string(smem) + " B of dynamic shared memory, above the " +
                                   std::to_string(max_dyn) + " B it may take on this device");
}

static std::mutex g_destroy_mu;   // orders a parent's deferred free against its children's destroys

// A parent destroyed while child contexts still borrow its tables keeps them until the last
// child is destroyed (its other calls are the caller's to stop).
extern "C" void exm_ctx_destroy(exm_ctx *ctx)
{
    if (!ctx) return;
    if (ctx->srv) exm_serve_destroy(ctx);   // its workers are children of this context
    exm_ctx *parent = ctx->parent, *free_parent = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_destroy_mu);
        if (!parent && ctx->n_children.load() > 0) {
            ctx->destroy_pending = true;
            return;
        }
        if (parent && parent->n_children.fetch_sub(1) == 1 && parent->destroy_pending) free_parent = parent;
    }
    ctx_free(ctx);
    if (free_parent) ctx_free(free_parent);
}

// the calling thread's last failure on a context (by the id of its message), and its last read
static std::atomic<uint64_t> g_errmsg_ids{1};
static thread_local uint64_t tl_err_owner = 0;
static thread_local std::string tl_err_msg, tl_err_read;

exm_errmsg::exm_errmsg() : id_(g_errmsg_ids.fetch_add(1)) {}

exm_errmsg &exm_errmsg::operator=(const std::string &m)
{
    {
        std::lock_guard<std::mutex> lk(mu_);
        msg_ = m;
    }
    tl_err_owner = id_;
    tl_err_msg = m;
    return *this;
}

exm_errmsg::operator std::string() const
{
    std::lock_guard<std::mutex> lk(mu_);
    return msg_;
}

const char *exm_errmsg::c_str() const
{
    if (tl_err_owner == id_) {
        tl_err_read = tl_err_msg;
    } else {
        std::lock_guard<std::mutex> lk(mu_);
        tl_err_read = msg_;
    }
    return tl_err_read.c_str();
}

extern "C" const char *exm_last_error(const exm_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

extern "C" size_t exm_ctx_bytes(const exm_ctx *ctx) { return ctx ? ctx->used : 0; }

// ------------------------------------------------------------------ store

extern "C" int exm_store_init(exm_ctx *ctx, int n_nodes, int ntau, int nphif, int nb, int nd, int dtype,
                              const int64_t *tau_idx, double beta0, double dbeta, double delta0, double ddelta)
{
    API_BEGIN(ctx)
    REQUIRE(!ctx->store_borrowed, EXM_ERR_STATE, "this context borrows its parent's store");
    REQUIRE(ctx->n_children.load() == 0, EXM_ERR_STATE, "child contexts borrow this store: destroy them first");
    EXM_CUDA(cudaSetDevice(ctx->dev));
    REQUIRE(n_nodes >= 1 && n_nodes <= EXM_MAX_NODES, EXM_ERR_ARG, "n_nodes must be 1..64");
    REQUIRE(ntau >= 1 && tau_idx, EXM_ERR_ARG, "need at least one lag");
    REQUIRE(nphif == EXM_NPHI / 2 + 1, EXM_ERR_ARG, "tables must hold NPHI/2 + 1 = 49 phase planes");
    REQUIRE(nb >= 2 && nb <= 4096 && nd >= 2 && nd <= 256, EXM_ERR_ARG, "need 2 <= nb <= 4096 and 2 <= nd <= 256");
    REQUIRE(dtype == EXM_DTYPE_F32 || dtype == EXM_DTYPE_F16 || dtype == EXM_DTYPE_BF16, EXM_ERR_ARG,
            "dtype must be EXM_DTYPE_F32, EXM_DTYPE_F16 or EXM_DTYPE_BF16");
    REQUIRE(dbeta > 0 && ddelta > 0, EXM_ERR_ARG, "grid steps must be positive");
    ctx->store_ok = ctx->prep_ok = false;
    ctx->tmap_ok = false;
    ctx->shard = false;
    ctx->s_before = 0.0;
    ctx->nn = n_nodes;
    ctx->ntau = ntau;
    ctx->nphif = nphif;
    ctx->nb = nb;
    ctx->nd = nd;
    const int al = (int)(16 / exm_dtype_bytes(dtype));   // elements per 16 bytes
    ctx->ndp = (nd + al - 1) / al * al;
    ctx->dtype = dtype;
    ctx->beta0 = beta0;
    ctx->dbeta = dbeta;
    ctx->delta0 = delta0;
    ctx->ddelta = ddelta;
    ctx->tau.assign(tau_idx, tau_idx + ntau);
    ctx->s.assign(n_nodes, 0.0);
    ctx->alo.assign(n_nodes, 0.0);
    ctx->ahi.assign(n_nodes, 0.0);
    ctx->node_set.assign(n_nodes, 0);
    ctx->tstride = (size_t)ntau * nphif * nb * ctx->ndp;
    exm_free(ctx, ctx->T);
    exm_alloc(ctx, ctx->T, ctx->tstride * n_nodes * exm_dtype_bytes(dtype));
    EXM_CUDA(cudaMemsetAsync(ctx->T.p, 0, ctx->T.bytes, ctx->stream));
    ctx->tscale.assign(n_nodes, 1.f);
    exm_ensure(ctx, ctx->d_tscale, sizeof(float) * EXM_MAX_NODES);
    EXM_CUDA(cudaMemcpyAsync(ctx->d_tscale.p, ctx->tscale.data(), sizeof(float) * n_nodes, cudaMemcpyHostToDevice,
                             ctx->stream));
    std::vector<int> t32(ntau);
    for (int r = 0; r < ntau; ++r) t32[r] = (int)tau_idx[r];
    exm_ensure(ctx, ctx->d_tau, sizeof(int) * ntau);
    EXM_CUDA(cudaMemcpy(ctx->d_tau.p, t32.data(), sizeof(int) * ntau, cudaMemcpyHostToDevice));
    exm_make_tmap(ctx);
    exm_ensure(ctx, ctx->d_stats, 4 * sizeof(unsigned long long));
    EXM_CUDA(cudaMemsetAsync(ctx->d_stats.p, 0, 4 * sizeof(unsigned long long), ctx->stream));
    EXM_CUDA(cudaStreamSynchronize(ctx->stream));
    API_END(ctx)
}

static void set_node_meta(exm_ctx *ctx, int k, double s, double alo, double ahi)
{
    REQUIRE(ctx->T.p, EXM_ERR_STATE, "exm_store_init first");
    REQUIRE(k >= 0 && k < ctx->nn, EXM_ERR_ARG, "node index out of range");
    REQUIRE(s > 0 && alo > 0 && ahi > alo, EXM_ERR_ARG, "node needs s > 0 and 0 < alpha_lo < alpha_hi");
    if (k > 0 && ctx->node_set[k - 1]) REQUIRE(s > ctx->s[k - 1], EXM_ERR_ARG, "nodes must be added with s ascending");
    ctx->s[k] = s;
    ctx->alo[k] = alo;
    ctx->ahi[k] = ahi;
    ctx->node_set[k] = 1;
    ctx->prep_ok = false;
    ctx->store_ok = std::all_of(ctx->node_set.begin(), ctx->node_set.end(), [](char c) { return c != 0; });
}

extern "C" int exm_store_set_node(exm_ctx *ctx, int k, double s, double alpha_lo, double alpha_hi, const float *T)
{
    API_BEGIN(ctx)
    REQUIRE(!ctx->store_borrowed, EXM_ERR_STATE, "this context borrows its parent's store");
    REQUIRE(ctx->n_children.load() == 0, EXM_ERR_STATE, "child contexts borrow this store: destroy them first");
    EXM_CUDA(cudaSetDevice(ctx->dev));
    REQUIRE(T, EXM_ERR_ARG, "null table");
    set_node_meta(ctx, k, s, alpha_lo, alpha_hi);
    const size_t rows = (size_t)ctx->ntau * ctx->nphif * ctx->nb;
    if (ctx->dtype == EXM_DTYPE_F32) {
        float *dst = (float *)ctx->T.p + (size_t)k * ctx->tstride;
        EXM_CUDA(cudaMemcpy2DAsync(dst, ctx->ndp * sizeof(float), T, ctx->nd * sizeof(float), ctx->nd * sizeof(float),
                                   rows, cudaMemcpyHostToDevice, ctx->stream));
    } else {   // the float32 node through a scratch copy, quantized on the device
        dbuf f;
        exm_alloc(ctx, f, sizeof(float) * rows * ctx->nd);
        EXM_CUDA(cudaMemcpyAsync(f.p, T, sizeof(float) * rows * ctx->nd, cudaMemcpyHostToDevice, ctx->stream));
        exm_store_quantize(ctx, k, (const float *)f.p, ctx->nd);
        exm_free(ctx, f);
    }
    EXM_CUDA(cudaStreamSynchronize(ctx->stream));
    API_END(ctx)
}

extern "C" int exm_store_load(exm_ctx *ctx, int first, int n, const char *const *paths, const int64_t *offsets,
                              const float *const *hosts, const double *s, const double *alpha_lo, const double *alpha_hi,
                              int readers, long long chunk_bytes, int flags, double *stats_out)
{
    API_BEGIN(ctx)
    REQUIRE(!ctx->store_borrowed, EXM_ERR_STATE, "this context borrows its parent's store");
    REQUIRE(ctx->n_children.load() == 0, EXM_ERR_STATE, "child contexts borrow this store: destroy them first");
    EXM_CUDA(cudaSetDevice(ctx->dev));
    REQUIRE(ctx->T.p, EXM_ERR_STATE, "exm_store_init first");
    REQUIRE(n >= 1 && first >= 0 && first + n <= ctx->nn, EXM_ERR_ARG, "node range outside the store");
    REQUIRE(s && alpha_lo && alpha_hi, EXM_ERR_ARG, "null node metadata");
    REQUIRE(paths || hosts, EXM_ERR_ARG, "neither files nor host tables");
    REQUIRE(!paths || offsets, EXM_ERR_ARG, "files without offsets");
    REQUIRE(readers >= 1 && readers <= 64, EXM_ERR_ARG, "readers must be 1..64");
    REQUIRE(chunk_bytes >= 0, EXM_ERR_ARG, "negative chunk size");
    REQUIRE((flags & ~EXM_LOAD_DIRECT) == 0, EXM_ERR_ARG, "unknown load flags");
    for (int i = 0; i < n; ++i) {
        REQUIRE(s[i] > 0 && alpha_lo[i] > 0 && alpha_hi[i] > alpha_lo[i], EXM_ERR_ARG,
                "node needs s > 0 and 0 < alpha_lo < alpha_hi");
        REQUIRE(i == 0 || s[i] > s[i - 1], EXM_ERR_ARG, "nodes must be added with s ascending");
    }
    if (first > 0 && ctx->node_set[first - 1]) REQUIRE(s[0] > ctx->s[first - 1], EXM_ERR_ARG, "nodes must be added with s ascending");
    exm_store_load_run(ctx, first, n, paths, offsets, hosts, readers, chunk_bytes, flags, stats_out);
    for (int i = 0; i < n; ++i) set_node_meta(ctx, first + i, s[i], alpha_lo[i], alpha_hi[i]);
    API_END(ctx)
}

extern "C" int exm_store_set_shard(exm_ctx *ctx, double s_before)
{
    API_BEGIN(ctx)
    REQUIRE(!ctx->store_borrowed, EXM_ERR_STATE, "this context borrows its parent's store");
    REQUIRE(ctx->n_children.load() == 0, EXM_ERR_STATE, "child contexts borrow this store: destroy them first");
    REQUIRE(ctx->T.p, EXM_ERR_STATE, "exm_store_init first");
    REQUIRE(s_before >= 0.0 && std::isfinite(s_before), EXM_ERR_ARG, "s_before must be finite and >= 0");
    REQUIRE(!ctx->node_set[0] || s_before < ctx->s[0], EXM_ERR_ARG, "s_before must lie below the shard's first node");
    ctx->shard = true;
    ctx->s_before = s_before;
    ctx->prep_ok = false;
    API_END(ctx)
}

extern "C" int exm_store_generate_node(exm_ctx *ctx, int k, double s, double alpha_lo, double alpha_hi, const float *M,
                                       const float *P, const float *Q, float S, uint32_t seed)
{
    API_BEGIN(ctx)
    REQUIRE(!ctx->store_borrowed, EXM_ERR_STATE, "this context borrows its parent's store");
    REQUIRE(ctx->n_children.load() == 0, EXM_ERR_STATE, "child contexts borrow this store: destroy them first");
    EXM_CUDA(cudaSetDevice(ctx->dev));
    REQUIRE(M && P && Q, EXM_ERR_ARG, "null generator factors");
    set_node_meta(ctx, k, s, alpha_lo, alpha_hi);
    exm_store_generate(ctx, k, M, P, Q, S, seed);
    API_END(ctx)
}

extern "C" int exm_store_get_node(exm_ctx *ctx, int k, float *T_out)
{
    API_BEGIN(ctx)
    EXM_CUDA(cudaSetDevice(ctx->dev));
    REQUIRE(ctx->T.p && k >= 0 && k < ctx->nn && T_out, EXM_ERR_ARG, "bad node or output");
    const size_t rows = (size_t)ctx->ntau * ctx->nphif * ctx->nb;
    if (ctx->dtype == EXM_DTYPE_F32) {
        const float *src = (const float *)ctx->T.p + (size_t)k * ctx->tstride;
        EXM_CUDA(cudaMemcpy2DAsync(T_out, ctx->nd * sizeof(float), src, ctx->ndp * sizeof(float),
                                   ctx->nd * sizeof(float), rows, cudaMemcpyDeviceToHost, ctx->stream));
        EXM_CUDA(cudaStreamSynchronize(ctx->stream));
    } else {   // the values scale * element, as float32
        dbuf f;
        exm_alloc(ctx, f, sizeof(float) * rows * ctx->nd);
        exm_store_dequantize(ctx, k, (float *)f.p, ctx->nd);
        EXM_CUDA(cudaMemcpyAsync(T_out, f.p, sizeof(float) * rows * ctx->nd, cudaMemcpyDeviceToHost, ctx->stream));
        EXM_CUDA(cudaStreamSynchronize(ctx->stream));
        exm_free(ctx, f);
    }
    API_END(ctx)
}

// ------------------------------------------------------------------ bank

extern "C" int exm_bank_set(exm_ctx *ctx, int nm, int nfreq, int lo, int n_time, const float *W, const double *u,
                            const double *M, const double *q, const double *chi)
{
    API_BEGIN(ctx)
    REQUIRE(nm >= 1 && nfreq >= 1 && lo >= 0 && n_time >= 2 && lo + nfreq <= n_time, EXM_ERR_ARG,
            "bank needs nm >= 1 and lo + nfreq <= n_time");
    REQUIRE(W && u && M && q && chi, EXM_ERR_ARG, "null bank array");
    ctx->nm = nm;
    ctx->nfreq = nfreq;
    ctx->lo = lo;
    ctx->nt = n_time;
    ctx->W.assign(W, W + (size_t)2 * nm * nfreq);
    ctx->u.assign(u, u + nm);
    ctx->M.assign(M, M + nm);
    ctx->q.assign(q, q + nm);
    ctx->chi.assign(chi, chi + nm);
    for (int m = 0; m < nm; ++m) REQUIRE(u[m] > 0, EXM_ERR_ARG, "template powers u must be positive");
    ctx->bank_ok = true;
    ctx->prep_ok = false;
    ctx->traj_ok = ctx->times_ok = false;
    API_END(ctx)
}

// ------------------------------------------------------------------ prepare: geometry, weights, cell weights

static std::vector<double> cell_weights(const exm_ctx *ctx)
{
    const int nm = ctx->nm;
    std::vector<double> cell(nm, 1.0);
    const std::vector<double> *axes[3] = {&ctx->M, &ctx->q, &ctx->chi};
    for (const auto *ax : axes) {
        std::vector<double> vals(*ax);
        std::sort(vals.begin(), vals.end());
        vals.erase(std::unique(vals.begin(), vals.end()), vals.end());
        const int n = (int)vals.size();
        if (n <= 1) continue;
        std::vector<double> g(n);
        g[0] = vals[1] - vals[0];
        g[n - 1] = vals[n - 1] - vals[n - 2];
        for (int i = 1; i < n - 1; ++i) g[i] = (vals[i + 1] - vals[i - 1]) / 2.0;
        for (int m = 0; m < nm; ++m) {
            const int j = (int)(std::lower_bound(vals.begin(), vals.end(), (*ax)[m]) - vals.begin());
            cell[m] *= g[j];
        }
    }
    double tot = 0.0;
    for (double c : cell) tot += c;
    for (double &c : cell) c /= tot;
    return cell;
}

template <typename T>
static void upload(exm_ctx *ctx, dbuf &b, const std::vector<T> &v)
{
    exm_ensure(ctx, b, sizeof(T) * std::max<size_t>(v.size(), 1));
    if (!v.empty()) EXM_CUDA(cudaMemcpy(b.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
}

// The n-point Gauss-Legendre rule on [-1, 1]: the nodes are the roots of the Legendre polynomial P_n, found by
// Newton's method from the asymptotic guesses cos(pi (i + 3/4) / (n + 1/2)) with P_n and P_n' from the
// three-term recurrence (k + 1) P_{k+1} = (2k + 1) x P_k - k P_{k-1}; the weights are 2 / ((1 - x^2) P_n'(x)^2).
// Symmetric pairs are computed once.
void exm_gauss_legendre_rule(int n, double *x, double *w)
{
    const double pi = 3.14159265358979323846;
    for (int i = 0; i < (n + 1) / 2; ++i) {
        double z = std::cos(pi * (i + 0.75) / (n + 0.5)), dp = 0.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = z;
            for (int k = 1; k < n; ++k) {
                const double p2 = ((2.0 * k + 1.0) * z * p1 - k * p0) / (k + 1.0);
                p0 = p1;
                p1 = p2;
            }
            dp = n * (z * p1 - p0) / (z * z - 1.0);
            const double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        double p0 = 1.0, p1 = z;
        for (int k = 1; k < n; ++k) {
            const double p2 = ((2.0 * k + 1.0) * z * p1 - k * p0) / (k + 1.0);
            p0 = p1;
            p1 = p2;
        }
        dp = n * (z * p1 - p0) / (z * z - 1.0);
        const double wi = 2.0 / ((1.0 - z * z) * dp * dp);
        x[n - 1 - i] = z;
        x[i] = -z;
        w[i] = w[n - 1 - i] = wi;
    }
}

extern "C" int exm_gauss_legendre(int n, double *x, double *w)
{
    if (n < 1 || n > 256 || !x || !w) return EXM_ERR_ARG;
    exm_gauss_legendre_rule(n, x, w);
    return EXM_OK;
}

extern "C" int exm_pe_prepare(exm_ctx *ctx, double ymin, int prior, const double *lny, const double *p_lny, int n_dens)
{
    API_BEGIN(ctx)
    EXM_CUDA(cudaSetDevice(ctx->dev));
    REQUIRE(ctx->store_ok, EXM_ERR_STATE, "store is not complete (exm_store_init + every node)");
    REQUIRE(ctx->bank_ok, EXM_ERR_STATE, "no bank (exm_bank_set)");
    const bool gl64 = (prior & EXM_QUAD_GL64) != 0;
    prior &= ~EXM_QUAD_GL64;
    REQUIRE(prior == EXM_PRIOR_VOLUME || (prior == EXM_PRIOR_TABULATED && lny && p_lny && n_dens >= 2), EXM_ERR_ARG,
            "the distance prior is 'volume' or a tabulated density");
    const int nn = ctx->nn, nm = ctx->nm;
    // node geometry, exmarg/search/pe.py:58-84, on the original template order
    std::vector<char> valid((size_t)nn * nm, 0);
    std::vector<double> y((size_t)(nn + 1) * nm, 0.0);
    std::vector<int> bnode(nm, -1);
    std::vector<double> blna(nm, 0.0);
    for (int k = 0; k < nn; ++k) {
        const double alo = std::min(ctx->alo[k], ymin * ymin);
        const double s_prev = k > 0 ? ctx->s[k - 1] : ctx->s_before;
        const double a_b = alo * (1.0 + 1e-9);
        for (int m = 0; m < nm; ++m) {
            const double a = ctx->s[k] / ctx->u[m];
            const bool o = (std::sqrt(a) >= ymin) && (a > alo) && (a < ctx->ahi[k]);
            valid[(size_t)k * nm + m] = o;
            y[(size_t)k * nm + m] = o ? std::sqrt(a) : 0.0;
            if (o && (s_prev / ctx->u[m] <= alo)) {
                bnode[m] = k;
                blna[m] = std::log(a_b);
                y[(size_t)nn * nm + m] = std::sqrt(a_b);
            }
        }
    }
    for (int m = 0; m < nm && !ctx->shard; ++m) {   // a shard's templates may reach its nodes 0 or 1 times
        int pts = 0;
        for (int k = 0; k <= nn; ++k) pts += y[(size_t)k * nm + m] > 0;
        if (pts < 2) {
            char buf[160];
            snprintf(buf, sizeof(buf), "template %d (M %.2f, u %.3f) reaches fewer than two store nodes", m,
                     ctx->M[m], ctx->u[m]);
            EXM_THROW(EXM_ERR_ARG, buf);
        }
    }
    // internal order: ascending u, so every node's valid templates form one range
    std::vector<int> order(nm);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return ctx->u[a] < ctx->u[b]; });
    ctx->order = order;
    ctx->mlo.assign(nn, 0);
    ctx->mhi.assign(nn, 0);
    for (int k = 0; k < nn; ++k) {
        int first = -1, last = -1;
        for (int i = 0; i < nm; ++i)
            if (valid[(size_t)k * nm + order[i]]) {
                if (first < 0) first = i;
                last = i;
            }
        if (first < 0) {
            ctx->mlo[k] = ctx->mhi[k] = 0;
            continue;
        }
        for (int i = first; i <= last; ++i)
            REQUIRE(valid[(size_t)k * nm + order[i]], EXM_ERR_ARG,
                    "node validity is not an interval in u (alpha limits vary across nodes)");
        ctx->mlo[k] = first;
        ctx->mhi[k] = last + 1;
    }
    std::vector<int> bn(nm);
    std::vector<double> boff(nm), cb(nm, 0.0), yint((size_t)(nn + 1) * nm), cellv = cell_weights(ctx), celli(nm);
    for (int i = 0; i < nm; ++i) {
        const int m = order[i];
        bn[i] = bnode[m];
        boff[i] = -std::log(ctx->u[m]) / ctx->dbeta;
        if (bnode[m] >= 0) cb[i] = (blna[m] - ctx->beta0) / ctx->dbeta + std::log(ctx->u[m]) / ctx->dbeta;
        for (int k = 0; k <= nn; ++k) yint[(size_t)k * nm + i] = y[(size_t)k * nm + m];
        celli[i] = cellv[m];
    }
    ctx->bnode = bn;
    ctx->ck.assign(nn, 0.0);
    std::vector<int> cki(EXM_MAX_NODES, 0);
    std::vector<double> ckd(EXM_MAX_NODES, 0.0);
    for (int k = 0; k < nn; ++k) {
        ctx->ck[k] = (std::log(ctx->s[k]) - ctx->beta0) / ctx->dbeta;
        ckd[k] = ctx->ck[k];
        cki[k] = (int)std::floor(ctx->ck[k]);
    }
    // W in internal order
    std::vector<float> Wi((size_t)2 * nm * ctx->nfreq);
    for (int i = 0; i < nm; ++i)
        memcpy(&Wi[(size_t)2 * i * ctx->nfreq], &ctx->W[(size_t)2 * order[i] * ctx->nfreq],
               sizeof(float) * 2 * ctx->nfreq);
    upload(ctx, ctx->d_W, Wi);
    upload(ctx, ctx->d_bhat_off, boff);
    upload(ctx, ctx->d_bnode, bn);
    upload(ctx, ctx->d_cb, cb);
    upload(ctx, ctx->d_cell, celli);
    upload(ctx, ctx->d_mlo, ctx->mlo);
    upload(ctx, ctx->d_mhi, ctx->mhi);
    upload(ctx, ctx->d_order, order);
    upload(ctx, ctx->d_cki, cki);
    upload(ctx, ctx->d_ckd, ckd);
    // distance-prior weights on the device
    dbuf dy, dd;
    upload(ctx, dy, yint);
    std::vector<double> dens;
    if (prior == EXM_PRIOR_TABULATED) {
        dens.assign(lny, lny + n_dens);
        dens.insert(dens.end(), p_lny, p_lny + n_dens);
    }
    upload(ctx, dd, dens);
    dbuf dg;
    if (gl64) {
        std::vector<double> g(128);
        exm_gauss_legendre_rule(64, g.data(), g.data() + 64);
        upload(ctx, dg, g);
    }
    exm_ensure(ctx, ctx->d_lnW, sizeof(double) * (size_t)(nn + 1) * nm);
    exm_run_distance_weights_y(ctx, (const double *)dy.p, ymin, prior, (const double *)dd.p,
                               (const double *)dd.p + (dens.empty() ? 0 : n_dens), n_dens,
                               gl64 ? (const double *)dg.p : nullptr);
    EXM_CUDA(cudaStreamSynchronize(ctx->stream));
    exm_free(ctx, dy);
    exm_free(ctx, dd);
    exm_free(ctx, dg);
    ctx->prep_ok = true;
    ctx->traj_ok = ctx->times_ok = false;
    API_END(ctx)
}

// ------------------------------------------------------------------ the per-segment pipeline

struct RunShape {
    int K, S, nwalk, use_sel, nmc_max, rc;
    float lw;
};

static RunShape run_shape(exm_ctx *ctx, int K, int S)
{
    RunShape rs;
    REQUIRE(K >= 0 && S >= 0, EXM_ERR_ARG, "n_loud and n_random must be >= 0");
    rs.K = K;
    rs.S = S;
    if (K > 0) {
        REQUIRE(S >= 1, EXM_ERR_ARG, "n_random must be >= 1 when n_loud > 0 (division by zero)");
        REQUIRE(ctx->nt - K >= 1, EXM_ERR_ARG, "high <= 0: n_loud must be below n_time");
        std::vector<int64_t> t = ctx->tau;
        std::sort(t.begin(), t.end());
        for (size_t i = 1; i < t.size(); ++i) REQUIRE(t[i] == t[i - 1] + 1, EXM_ERR_ARG, "lags are not contiguous");
        rs.nwalk = K + S;
        rs.use_sel = 1;
        rs.lw = (float)std::log((double)(ctx->nt - K) / (double)S);
    } else {
        rs.nwalk = ctx->nt;
        rs.use_sel = 0;
        rs.lw = 0.f;
    }
    rs.nmc_max = std::min(ctx->nm, EXM_MAX_CHUNK);
    const size_t per_lag = (size_t)rs.nmc_max * rs.nwalk * 20;
    const size_t cap = (size_t)8 << 30;
    rs.rc = (int)std::max<size_t>(1, std::min<size_t>((size_t)ctx->ntau, cap / std::max<size_t>(per_lag, 1)));
    return rs;
}

static void ensure_slot(exm_ctx *ctx, exm_slot &sl, const RunShape &rs)
{
    const size_t nmc = rs.nmc_max, nt = ctx->nt, nf = ctx->nfreq;
    exm_ensure(ctx, sl.traj, 2 * nmc * nt * sizeof(float2));
    if (ctx->traj_fp64) exm_ensure(ctx, sl.trajlo, 2 * nmc * nt * sizeof(float));
    exm_ensure(ctx, sl.fft, 2 * nmc * nt * sizeof(double2));
    const size_t n_draws = rs.K > 0 ? (((size_t)ctx->nm * rs.S + EXM_MAX_REJ + 63) / 64) * 64 : 0;
    exm_ensure(ctx, sl.keys, std::max<size_t>(rs.K > 0 ? nmc * nt : 1, n_draws) * sizeof(uint32_t));
    exm_ensure(ctx, sl.picks, std::max<size_t>(1, (size_t)ctx->nm * rs.S) * sizeof(int32_t));
    exm_ensure(ctx, sl.rej, (1 + EXM_MAX_REJ) * sizeof(int));
    exm_ensure(ctx, sl.sel, std::max<size_t>(1, rs.use_sel ? nmc * rs.nwalk : 1) * sizeof(int32_t));
    exm_ensure(ctx, sl.hist, (EXM_HB_N + 256) * sizeof(int));
    exm_ensure(ctx, sl.win, (2 + EXM_MAX_NODES) * sizeof(int));
    exm_ensure(ctx, sl.cnt, (size_t)rs.rc * EXM_NPAIR * (nmc + 1) * sizeof(int));
    const size_t pitch = (size_t)exm_desc_pitch((long long)nmc * rs.nwalk);
    exm_ensure(ctx, sl.desc, (size_t)rs.rc * pitch * sizeof(uint4));
    exm_ensure(ctx, sl.tside, (size_t)rs.rc * pitch * sizeof(int32_t));
    exm_ensure(ctx, sl.part, (size_t)(ctx->nn + 1) * ctx->ntau * ctx->nm * sizeof(double));
    exm_ensure(ctx, sl.lnl, (size_t)ctx->nm * sizeof(double));
    exm_ensure(ctx, sl.lnb, sizeof(double));
    exm_ensure(ctx, sl.dev_err, sizeof(unsigned));
    exm_ensure(ctx, sl.din, 6 * nf * sizeof(double) + 2 * nf * sizeof(float2) + 4 * sizeof(uint64_t));
    const size_t hin = 6 * nf * sizeof(double) + 4 * sizeof(uint64_t);
    if (!sl.hostin.p || sl.hostin.bytes < hin) {
        if (sl.hostin.p) cudaFreeHost(sl.hostin.p);
        sl.hostin.p = nullptr;
        EXM_CUDA(cudaMallocHost(&sl.hostin.p, hin));
        sl.hostin.bytes = hin;
    }
}

// the segment's data and the PCG64 state of its seed into the pinned staging buffer
static void stage_host(exm_ctx *ctx, exm_slot &sl, const double *dH, const double *dL, const double *s2H,
                       const double *s2L, uint64_t seed)
{
    const size_t nf = ctx->nfreq;
    double *h = (double *)sl.hostin.p;
    memcpy(h, dH, 2 * nf * sizeof(double));
    memcpy(h + 2 * nf, dL, 2 * nf * sizeof(double));
    memcpy(h + 4 * nf, s2H, nf * sizeof(double));
    memcpy(h + 5 * nf, s2L, nf * sizeof(double));
    exm_pcg_words(seed, (uint64_t *)(h + 6 * nf));
}

// the staged input to the device (a stream operation: part of a captured graph)
static void copy_input(exm_ctx *ctx, exm_slot &sl)
{
    const size_t nf = ctx->nfreq;
    EXM_CUDA(cudaMemcpyAsync(sl.din.p, sl.hostin.p, 6 * nf * sizeof(double) + 4 * sizeof(uint64_t),
                             cudaMemcpyHostToDevice, ctx->stream));
}

static const uint64_t *state_words(exm_ctx *ctx, exm_slot &sl)
{
    return (const uint64_t *)((const double *)sl.din.p + 6 * (size_t)ctx->nfreq);
}

static void stage_input(exm_ctx *ctx, exm_slot &sl, const double *dH, const double *dL, const double *s2H,
                        const double *s2L, uint64_t seed = 0)
{
    stage_host(ctx, sl, dH, dL, s2H, s2L, seed);
    copy_input(ctx, sl);
}

static void check_dev_err(exm_ctx *ctx, exm_slot &sl)
{
    unsigned e = 0;
    EXM_CUDA(cudaMemcpyAsync(&e, sl.dev_err.p, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    EXM_CUDA(cudaStreamSynchronize(ctx->stream));
    if (e & EXM_DEVERR_TIMEOUT)
        EXM_THROW(EXM_ERR_TIMEOUT, "a bounded device wait (TMA copy of a table plane) ran out");
    if (e & EXM_DEVERR_BOUNDS) EXM_THROW(EXM_ERR_CUDA, "a tap descriptor pointed outside its block (internal error)");
}

// NVTX range of one pipeline stage on the calling host thread (the launches it encloses show up under it in
// a timeline profiler); free when no profiler is attached
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

// everything of one segment from the staged input to lnl / lnb on the device
static void run_segment(exm_ctx *ctx, exm_slot &sl, const RunShape &rs)
{
    NvtxRange seg_range("exm segment");
    const int tt = exm_tim_begin(ctx, 0);
    EXM_CUDA(cudaMemsetAsync(sl.dev_err.p, 0, sizeof(unsigned), ctx->stream));
    if (rs.K > 0) {
        NvtxRange nr("exm select: random draws");
        const int h = exm_tim_begin(ctx, 2);
        exm_run_pcg(ctx, sl, state_words(ctx, sl), rs.K, rs.S);
        exm_tim_end(ctx, h);
    }
    for (int m_base = 0; m_base < ctx->nm; m_base += rs.nmc_max) {
        const int nmc = std::min(rs.nmc_max, ctx->nm - m_base);
        int h;
        {
            NvtxRange nr("exm filter");
            h = exm_tim_begin(ctx, 1);
            exm_run_filter(ctx, sl, (const float2 *)ctx->d_W.p + (size_t)m_base * ctx->nfreq, nmc);
            exm_tim_end(ctx, h);
        }
        if (rs.K > 0) {
            NvtxRange nr("exm select");
            h = exm_tim_begin(ctx, 2);
            exm_run_topk(ctx, sl, nmc, (const int *)ctx->d_order.p + m_base, rs.K, rs.S);
            exm_tim_end(ctx, h);
        }
        ChunkInfo ci{m_base, nmc, rs.nwalk, rs.use_sel, rs.lw};
        for (int r0 = 0; r0 < ctx->ntau; r0 += rs.rc) {
            const int rc = std::min(rs.rc, ctx->ntau - r0);
            {
                NvtxRange nr("exm taps");
                h = exm_tim_begin(ctx, 3);
                exm_run_taps(ctx, sl, ci, r0, rc, r0 == 0);
                exm_tim_end(ctx, h);
            }
            NvtxRange nr("exm gather");
            h = exm_tim_begin(ctx, 4);
            exm_run_gather_planes(ctx, sl, ci, r0, rc);
            exm_tim_end(ctx, h);
        }
        NvtxRange nr("exm epilogue");
        h = exm_tim_begin(ctx, 5);
        exm_run_node_lse(ctx, sl, m_base, nmc);
        exm_tim_end(ctx, h);
    }
    NvtxRange nr("exm epilogue: ln B");
    const int h = exm_tim_begin(ctx, 5);
    exm_run_lnb(ctx, sl);
    exm_tim_end(ctx, h);
    exm_tim_end(ctx, tt);
    ctx->segments += 1;
}

// the whole per-segment device sequence (input copy included) as one CUDA graph, captured on
// first use for the current shape and buffers and replayed for every later segment
static void run_segment_graph(exm_ctx *ctx, exm_slot &sl, const RunShape &rs)
{
    const long long key[6] = {ctx->nm, ctx->nt, rs.K, rs.S, ctx->gather_cfg, ctx->alloc_gen};
    if (!ctx->graph_exec || memcmp(key, ctx->graph_key, sizeof(key)) != 0) {
        if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
        ctx->graph_exec = nullptr;
        // this segment runs uncaptured: plans, work areas, kernel modules and their attributes
        // are all in place before the capture, which then records the same launches for the
        // following segments
        copy_input(ctx, sl);
        run_segment(ctx, sl, rs);
        EXM_CUDA(cudaStreamSynchronize(ctx->stream));
        const long long gen0 = ctx->alloc_gen;
        const bool tim = ctx->tim_on;
        const double taps0 = ctx->node_taps, tlw0 = ctx->tlw, seg0 = ctx->segments;
        const long long l0 = ctx->launches, g0 = ctx->gather_launches;
        ctx->tim_on = false;
        cudaGraph_t g = nullptr;
        EXM_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        try {
            copy_input(ctx, sl);
            run_segment(ctx, sl, rs);
        } catch (...) {
            cudaStreamEndCapture(ctx->stream, &g);
            if (g) cudaGraphDestroy(g);
            ctx->tim_on = tim;
            throw;
        }
        EXM_CUDA(cudaStreamEndCapture(ctx->stream, &g));
        ctx->tim_on = tim;
        if (ctx->alloc_gen != gen0) {   // something was allocated while capturing: buffers not stable
            cudaGraphDestroy(g);
            EXM_THROW(EXM_ERR_STATE, "workspace changed while capturing the segment graph");
        }
        cudaError_t e = cudaGraphInstantiate(&ctx->graph_exec, g, 0);
        cudaGraphDestroy(g);
        EXM_CUDA(e);
        ctx->graph_node_taps = ctx->node_taps - taps0;
        ctx->graph_tlw = ctx->tlw - tlw0;
        ctx->graph_launches = ctx->launches - l0;
        ctx->graph_gathers = ctx->gather_launches - g0;
        ctx->node_taps = taps0;   // counted per replay below
        ctx->tlw = tlw0;
        ctx->segments = seg0;
        ctx->launches = l0;
        ctx->gather_launches = g0;
        memcpy(ctx->graph_key, key, sizeof(key));
        return;
    }
    NvtxRange nr("exm segment (graph replay)");
    const int h = exm_tim_begin(ctx, 0);
    EXM_CUDA(cudaGraphLaunch(ctx->graph_exec, ctx->stream));
    exm_tim_end(ctx, h);
    ctx->node_taps += ctx->graph_node_taps;
    ctx->tlw += ctx->graph_tlw;
    ctx->launches += ctx->graph_launches;
    ctx->gather_launches += ctx->graph_gathers;
    ctx->segments += 1;
}

extern "C" int exm_pe_intrinsic(exm_ctx *ctx, int n_seg, const double *d_H, const double *d_L, const double *sig2_H,
                                const double *sig2_L, const int64_t *seeds, int n_loud, int n_random,
                                double *ln_lambda, double *ln_b)
{
    API_BEGIN(ctx)
    EXM_CUDA(cudaSetDevice(ctx->dev));
    REQUIRE(ctx->prep_ok, EXM_ERR_STATE, "exm_pe_prepare first");
    REQUIRE(!ctx->shard, EXM_ERR_STATE, "a store shard gives node values (exm_node_values); ln Lambda needs every shard's");
    REQUIRE(n_seg >= 0 && d_H && d_L && sig2_H && sig2_L && ln_lambda && ln_b, EXM_ERR_ARG, "null argument");
    REQUIRE(n_loud == 0 || seeds, EXM_ERR_ARG, "seeds are needed when n_loud > 0");
    const RunShape rs = run_shape(ctx, n_loud, n_random);
    exm_slot &sl = ctx->slot;
    ensure_slot(ctx, sl, rs);
    std::vector<double> lnl(ctx->nm);
    const size_t nf = ctx->nfreq;
    const bool graph = ctx->use_graph && ctx->nm <= rs.nmc_max && rs.rc >= ctx->ntau;
    for (int e = 0; e < n_seg; ++e) {
        REQUIRE(rs.K == 0 || seeds[e] >= 0, EXM_ERR_ARG, "seed must be non-negative");
        const uint64_t seed = rs.K > 0 ? (uint64_t)seeds[e] : 0;
        if (graph) {
            stage_host(ctx, sl, d_H + (size_t)e * 2 * nf, d_L + (size_t)e * 2 * nf, sig2_H, sig2_L, seed);
            run_segment_graph(ctx, sl, rs);
        } else {
            stage_input(ctx, sl, d_H + (size_t)e * 2 * nf, d_L + (size_t)e * 2 * nf, sig2_H, sig2_L, seed);
            run_segment(ctx, sl, rs);
        }
        EXM_CUDA(cudaMemcpyAsync(lnl.data(), sl.lnl.p, sizeof(double) * ctx->nm, cudaMemcpyDeviceToHost, ctx->stream));
        EXM_CUDA(cudaMemcpyAsync(ln_b + e, sl.lnb.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        check_dev_err(ctx, sl);
        exm_tim_collect(ctx);
        for (int i = 0; i < ctx->nm; ++i) ln_lambda[(size_t)e * ctx->nm + ctx->order[i]] = lnl[i];
    }
    ctx->traj_ok = ctx->times_ok = false;
    ctx->last_shape_ok = n_seg > 0;
    API_END(ctx)
}

// ------------------------------------------------------------------ autotuner

extern "C" int exm_autotune(exm_ctx *ctx, int n_loud, int n_random, int reps, int *best_cfg, int *best_chunk_pct,
                            double *ms_per_cfg)
{
    API_BEGIN(ctx)
    EXM_CUDA(cudaSetDevice(ctx->dev));
    REQUIRE(ctx->prep_ok, EXM_ERR_STATE, "exm_pe_prepare first");
    REQUIRE(ctx->last_shape_ok, EXM_ERR_STATE, "run exm_pe_intrinsic once first (the autotuner replays its last segment)");
    const RunShape rs = run_shape(ctx, n_loud, n_random);
    REQUIRE(rs.nmc_max >= ctx->nm && rs.rc >= ctx->ntau, EXM_ERR_ARG,
            "the autotuner needs the whole bank and every lag in one gather (bank <= 8192 templates)");
    exm_slot &sl = ctx->slot;
    ChunkInfo ci{0, ctx->nm, rs.nwalk, rs.use_sel, rs.lw};
    const int n = exm_gather_num_cfgs();
    cudaEvent_t e0, e1;
    EXM_CUDA(cudaEventCreate(&e0));
    EXM_CUDA(cudaEventCreate(&e1));
    const int keep = ctx->gather_cfg;
    const bool tim = ctx->tim_on;
    ctx->tim_on = false;
    auto time_gather = [&]() {
        exm_run_gather_planes(ctx, sl, ci, 0, ctx->ntau);   // warm-up (and function attributes)
        EXM_CUDA(cudaEventRecord(e0, ctx->stream));
        for (int r = 0; r < std::max(1, reps); ++r) exm_run_gather_planes(ctx, sl, ci, 0, ctx->ntau);
        EXM_CUDA(cudaEventRecord(e1, ctx->stream));
        EXM_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        EXM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        return ms / std::max(1, reps);
    };
    // 1: every launch shape with the default template chunk
    double best = 1e300;
    int arg = keep;
    ctx->gather_chunk_pct = 100;
    for (int c = 0; c < n; ++c) {
        ctx->gather_cfg = c;
        const double per = time_gather();
        if (ms_per_cfg) ms_per_cfg[c] = per;
        if (per < best) {
            best = per;
            arg = c;
        }
    }
    // 2: the templates per gather block (percent of the one-wave-per-lag size) with the best shape
    static const int pcts[] = {50, 150, 200};
    int best_pct = 100;
    ctx->gather_cfg = arg;
    for (int i = 0; i < 3; ++i) {
        ctx->gather_chunk_pct = pcts[i];
        const double per = time_gather();
        if (ms_per_cfg) ms_per_cfg[n + i] = per;
        if (per < best) {
            best = per;
            best_pct = pcts[i];
        }
    }
    ctx->gather_chunk_pct = best_pct;
    ctx->tim_on = tim;
    ctx->gather_cfg = arg;
    if (best_cfg) *best_cfg = arg;
    if (best_chunk_pct) *best_chunk_pct = best_pct;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    check_dev_err(ctx, sl);
    API_END(ctx)
}

extern "C" int exm_set_gather_cfg(exm_ctx *ctx, int cfg, int chunk_pct)
{
    API_BEGIN(ctx)
    REQUIRE(cfg >= 0 && cfg < exm_gather_num_cfgs(), EXM_ERR_ARG, "no such gather launch shape");
    REQUIRE(chunk_pct == 0 || (chunk_pct >= 10 && chunk_pct <= 1000), EXM_ERR_ARG,
            "chunk_pct must be 0 (keep) or 10..1000");
    ctx->gather_cfg = cfg;
    if (chunk_pct) ctx->gather_chunk_pct = chunk_pct;
    API_END(ctx)
}

// ------------------------------------------------------------------ stage entry points

static RunShape stage_shape(exm_ctx *ctx, int K, int S)
{
    REQUIRE(ctx->prep_ok, EXM_ERR_STATE, "exm_pe_prepare first");
    REQUIRE(ctx->nm <= EXM_MAX_CHUNK, EXM_ERR_ARG, "stage entry points take banks of at most 8192 templates");
    return run_shape(ctx, K, S);
}

extern "C" int exm_filter(exm_ctx *ctx, const double *d_H, const double *d_L, const double *sig2_H,
                          const double *sig2_L, float *traj_out)
{
    API_BEGIN(ctx)
    EXM_CUDA(cudaSetDevice(ctx->dev));
    RunShape rs = stage_shape(ctx, 0, 0);
    exm_slot &sl = ctx->slot;
    ensure_slot(ctx, sl, rs);
    stage_input(ctx, sl, d_H, d_L, sig2_H, sig2_L);
    exm_run_filter(ctx, sl, (const float2 *)ctx->d_W.p, ctx->nm);
    EXM_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->traj_ok = true;
    ctx->times_ok = false;
    ctx->cur_nwalk = ctx->nt;
    ctx->cur_lw = 0.f;
    if (traj_out) {
        const size_t nt = ctx->nt, nm = ctx->nm;
        std::vector<float2> h(2 * nm * nt);
        EXM_CUDA(cudaMemcpy(h.data(), sl.traj.p, sizeof(float2) * h.size(), cudaMemcpyDeviceToHost));
        for (int det = 0; det < 2; ++det)
            for (size_t i = 0; i < nm; ++i) {
                const size_t m = ctx->order[i];
                const float2 *src = &h[(det * nm + i) * nt];
                float *lq = traj_out + ((size_t)(2 * det) * nm + m) * nt;
                float *ph = traj_out + ((size_t)(2 * det + 1) * nm + m) * nt;
                for (size_t t = 0; t < nt; ++t) {
                    lq[t] = src[t].x;
                    ph[t] = src[t].y;
                }
            }
    }
    API_END(ctx)
}

extern "C" int exm_set_trajectories(exm_ctx *ctx, const float *traj)
{
    API_BEGIN(ctx)
    EXM_CUDA(cudaSetDevice(ctx->dev));
    REQUIRE(traj, EXM_ERR_ARG, "null trajectories");
    RunShape rs = stage_shape(ctx, 0, 0);
    exm_slot &sl = ctx->slot;
    ensure_slot(ctx, sl, rs);
    const size_t nt = ctx->nt, nm = ctx->nm;
    std::vector<float2> h(2 * nm * nt);
    for (int det = 0; det < 2; ++det)
        for (size_t i = 0; i < nm; ++i) {
            const size_t m = ctx->order[i];
            const float *lq = traj + ((size_t)(2 * det) * nm + m) * nt;
            const float *ph = traj + ((size_t)(2 * det + 1) * nm + m) * nt;
            float2 *dst = &h[(det * nm + i) * nt];
            for (size_t t = 0; t < nt; ++t) dst[t] = make_float2(lq[t], ph[t]);
        }
    EXM_CUDA(cudaMemcpy(sl.traj.p, h.data(), sizeof(float2) * h.size(), cudaMemcpyHostToDevice));
    if (sl.trajlo.p)   // float32 trajectories: no residual
        EXM_CUDA(cudaMemset(sl.trajlo.p, 0, std::min(sl.trajlo.bytes, sizeof(float) * h.size())));
    ctx->traj_ok = true;
    ctx->times_ok = false;
    ctx->cur_nwalk = ctx->nt;
    ctx->cur_lw = 0.f;
    API_END(ctx)
}

extern "C" int exm_select_times(exm_ctx *ctx, int64_t seed, int n_loud, int n_random, int32_t *sel_out, float *lw_out)
{
    API_BEGIN(ctx)
    EXM_CUDA(cudaSetDevice(ctx->dev));
    REQUIRE(ctx->traj_ok, EXM_ERR_STATE, "no trajectories (exm_filter or exm_set_trajectories first)");
    REQUIRE(n_loud > 0, EXM_ERR_ARG, "select_times needs n_loud > 0");
    REQUIRE(seed >= 0, EXM_ERR_ARG, "seed must be non-negative");
    RunShape rs = stage_shape(ctx, n_loud, n_random);
    exm_slot &sl = ctx->slot;
    ensure_slot(ctx, sl, rs);
    uint64_t *w = (uint64_t *)((double *)sl.hostin.p + 6 * (size_t)ctx->nfreq);
    exm_pcg_words((uint64_t)seed, w);
    EXM_CUDA(cudaMemcpyAsync((void *)state_words(ctx, sl), w, 4 * sizeof(uint64_t), cudaMemcpyHostToDevice,
                             ctx->stream));
    exm_run_pcg(ctx, sl, state_words(ctx, sl), rs.K, rs.S);
    exm_run_topk(ctx, sl, ctx->nm, (const int *)ctx->d_order.p, rs.K, rs.S);
    EXM_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->times_ok = true;
    ctx->cur_nwalk = rs.nwalk;
    ctx->cur_lw = rs.lw;
    if (sel_out || lw_out) {
        const size_t nw = rs.nwalk, nm = ctx->nm;
        std::vector<int32_t> h(nm * nw);
        EXM_CUDA(cudaMemcpy(h.data(), sl.sel.p, sizeof(int32_t) * h.size(), cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < nm; ++i) {
            const size_t m = ctx->order[i];
            for (size_t w = 0; w < nw; ++w) {
                const int32_t v = h[i * nw + w];
                if (sel_out) sel_out[m * nw + w] = v & 0x7FFFFFFF;
                if (lw_out) lw_out[m * nw + w] = (v < 0) ? rs.lw : 0.f;
            }
        }
    }
    API_END(ctx)
}

extern "C" int exm_ctx_set_filter_precision(exm_ctx *ctx, int mode)
{
    API_BEGIN(ctx)
    REQUIRE(mode == EXM_FILTER_REFERENCE || mode == EXM_FILTER_FP64, EXM_ERR_ARG,
            "filter precision is EXM_FILTER_REFERENCE or EXM_FILTER_FP64");
    ctx->traj_fp64 = mode == EXM_FILTER_FP64;
    ctx->traj_ok = ctx->times_ok = false;   // trajectories of the other precision are not reused
    ctx->graph_key[0] = -1;
    API_END(ctx)
}

extern "C" int exm_ctx_test_wait_expiry(exm_ctx *ctx, int enable)
{
    API_BEGIN(ctx)
    ctx->test_wait_expiry = enable != 0;
    ctx->graph_key[0] = -1;   // a captured graph holds the old launch arguments
    API_END(ctx)
}

extern "C" int exm_np_exp32(exm_ctx *ctx, const float *x, float *y, int64_t n)
{
    API_BEGIN(ctx)
    EXM_CUDA(cudaSetDevice(ctx->dev));
    REQUIRE(n >= 0 && (n == 0 || (x && y)), EXM_ERR_ARG, "bad exp arguments");
    if (n == 0) return EXM_OK;
    dbuf dx;
    exm_alloc(ctx, dx, sizeof(float) * 2 * (size_t)n);
    float *d_x = (float *)dx.p, *d_y = d_x + n;
    EXM_CUDA(cudaMemcpyAsync(d_x, x, sizeof(float) * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    exm_run_np_exp32(ctx, d_x, d_y, (long long)n);
    EXM_CUDA(cudaMemcpyAsync(y, d_y, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
    EXM_CUDA(cudaStreamSynchronize(ctx->stream));
    exm_free(ctx, dx);
    API_END(ctx)
}

extern "C" int exm_set_times(exm_ctx *ctx, int nwalk, const int32_t *sel, const float *lw)
{
    API_BEGIN(ctx)
    EXM_CUDA(cudaSetDevice(ctx->dev));
    REQUIRE(ctx->traj_ok, EXM_ERR_STATE, "no trajectories");
    REQUIRE(nwalk >= 0, EXM_ERR_ARG, "nwalk must be >= 0");
    if (nwalk == 0) {
        ctx->times_ok = false;
        ctx->cur_nwalk = ctx->nt;
        ctx->cur_lw = 0.f;
        return EXM_OK;
    }
    REQUIRE(sel && lw, EXM_ERR_ARG, "null times");
    const size_t nm = ctx->nm;
    float lwv = 0.f;
    std::vector<int32_t> h(nm * nwalk);
    for (size_t i = 0; i < nm; ++i) {
        const size_t m = ctx->order[i];
        for (int w = 0; w < nwalk; ++w) {
            const int32_t t = sel[m * nwalk + w];
            const float l = lw[m * nwalk + w];
            REQUIRE(t >= 0 && t < ctx->nt, EXM_ERR_ARG, "time index out of range");
            if (l != 0.f) {
                REQUIRE(lwv == 0.f || lwv == l, EXM_ERR_ARG, "every drawn time must carry the same log weight");
                lwv = l;
            }
            h[i * nwalk + w] = t | (l != 0.f ? (int32_t)0x80000000 : 0);
        }
    }
    RunShape rs = stage_shape(ctx, 0, 0);
    rs.nwalk = nwalk;
    rs.use_sel = 1;
    exm_slot &sl = ctx->slot;
    exm_ensure(ctx, sl.sel, sizeof(int32_t) * h.size());
    EXM_CUDA(cudaMemcpy(sl.sel.p, h.data(), sizeof(int32_t) * h.size(), cudaMemcpyHostToDevice));
    ctx->times_ok = true;
    ctx->cur_nwalk = nwalk;
    ctx->cur_lw = lwv;
    API_END(ctx)
}

extern "C" int exm_gather(exm_ctx *ctx, int nsel, int ns, const int64_t *mass_ids, const double *lna,
                          const int64_t *tab_ids, double *out)
{
    API_BEGIN(ctx)
    EXM_CUDA(cudaSetDevice(ctx->dev));
    REQUIRE(ctx->traj_ok, EXM_ERR_STATE, "no trajectories");
    REQUIRE(nsel >= 1 && ns >= 1 && mass_ids && lna && tab_ids && out, EXM_ERR_ARG, "bad gather arguments");
    std::vector<int> rows(nsel), tab((size_t)nsel * ns);
    std::vector<int> rank(ctx->nm);
    for (int i = 0; i < ctx->nm; ++i) rank[ctx->order[i]] = i;
    for (int j = 0; j < nsel; ++j) {
        REQUIRE(mass_ids[j] >= 0 && mass_ids[j] < ctx->nm, EXM_ERR_ARG, "mass id out of range");
        rows[j] = rank[mass_ids[j]];
        for (int n = 0; n < ns; ++n) {
            const int64_t t = tab_ids[(size_t)j * ns + n];
            REQUIRE(t >= 0 && t < ctx->nn, EXM_ERR_ARG, "table id out of range");
            tab[(size_t)j * ns + n] = (int)t;
        }
    }
    exm_slot &sl = ctx->slot;
    dbuf drows, dtab, dlna, dout;
    upload(ctx, drows, rows);
    upload(ctx, dtab, tab);
    std::vector<double> l(lna, lna + (size_t)nsel * ns);
    upload(ctx, dlna, l);
    exm_alloc(ctx, dout, sizeof(double) * (size_t)nsel * ns);
    exm_ensure(ctx, sl.part, std::max(sl.part.bytes, sizeof(double) * 2 * (size_t)ns * ctx->ntau * nsel));
    exm_run_gather_simple(ctx, sl, nsel, ns, (const int *)drows.p, (const int *)dtab.p, (const double *)dlna.p,
                          ctx->times_ok ? ctx->cur_nwalk : ctx->nt, ctx->times_ok ? 1 : 0, ctx->cur_lw,
                          (double *)dout.p);
    EXM_CUDA(cudaMemcpyAsync(out, dout.p, sizeof(double) * (size_t)nsel * ns, cudaMemcpyDeviceToHost, ctx->stream));
    EXM_CUDA(cudaStreamSynchronize(ctx->stream));
    exm_free(ctx, drows);
    exm_free(ctx, dtab);
    exm_free(ctx, dlna);
    exm_free(ctx, dout);
    API_END(ctx)
}

extern "C" int exm_node_values(exm_ctx *ctx, double *lamN_out)
{
    API_BEGIN(ctx)
    EXM_CUDA(cudaSetDevice(ctx->dev));
    REQUIRE(ctx->traj_ok, EXM_ERR_STATE, "no trajectories");
    REQUIRE(lamN_out, EXM_ERR_ARG, "null output");
    RunShape rs = stage_shape(ctx, 0, 0);
    rs.nwalk = ctx->times_ok ? ctx->cur_nwalk : ctx->nt;
    rs.use_sel = ctx->times_ok ? 1 : 0;
    rs.lw = ctx->cur_lw;
    const size_t per_lag = (size_t)ctx->nm * rs.nwalk * 20;
    rs.rc = (int)std::max<size_t>(1, std::min<size_t>((size_t)ctx->ntau, ((size_t)8 << 30) / per_lag));
    exm_slot &sl = ctx->slot;
    exm_ensure(ctx, sl.cnt, (size_t)rs.rc * EXM_NPAIR * (ctx->nm + 1) * sizeof(int));
    const size_t pitch = (size_t)exm_desc_pitch((long long)ctx->nm * rs.nwalk);
    exm_ensure(ctx, sl.desc, (size_t)rs.rc * pitch * sizeof(uint4));
    exm_ensure(ctx, sl.tside, (size_t)rs.rc * pitch * sizeof(int32_t));
    exm_ensure(ctx, sl.part, (size_t)(ctx->nn + 1) * ctx->ntau * ctx->nm * sizeof(double));
    EXM_CUDA(cudaMemsetAsync(sl.dev_err.p, 0, sizeof(unsigned), ctx->stream));
    ChunkInfo ci{0, ctx->nm, rs.nwalk, rs.use_sel, rs.lw};
    for (int r0 = 0; r0 < ctx->ntau; r0 += rs.rc) {
        const int rc = std::min(rs.rc, ctx->ntau - r0);
        exm_run_taps(ctx, sl, ci, r0, rc, r0 == 0);
        exm_run_gather_planes(ctx, sl, ci, r0, rc);
    }
    dbuf dl;
    exm_alloc(ctx, dl, sizeof(double) * (size_t)(ctx->nn + 1) * ctx->nm);
    exm_run_node_values(ctx, sl, (double *)dl.p);
    std::vector<double> h((size_t)(ctx->nn + 1) * ctx->nm);
    EXM_CUDA(cudaMemcpyAsync(h.data(), dl.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, ctx->stream));
    check_dev_err(ctx, sl);
    exm_free(ctx, dl);
    for (int k = 0; k <= ctx->nn; ++k)
        for (int i = 0; i < ctx->nm; ++i) lamN_out[(size_t)k * ctx->nm + ctx->order[i]] = h[(size_t)k * ctx->nm + i];
    API_END(ctx)
}
