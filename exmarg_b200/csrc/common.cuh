// Shared definitions of libexmarg_b200: the context, device-memory accounting,
// error reporting and the constants of the table geometry.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/exmarg_b200.h"

#define EXM_NPHI 96     // phase bins of the full circle (exmarg/search/gather.py:29)
#define EXM_NPAIR 48    // plane pairs (p, p+1), p = 0..47, of the 49 stored phase planes

// ------------------------------------------------------------------ errors

struct exm_error {
    int code;
    std::string msg;
};

#define EXM_THROW(code, msg) throw exm_error{(code), (msg)}
#define EXM_CUDA(call)                                                                              \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            throw exm_error{EXM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)};      \
    } while (0)
#define EXM_CUFFT(call)                                                                             \
    do {                                                                                            \
        cufftResult r_ = (call);                                                                    \
        if (r_ != CUFFT_SUCCESS)                                                                    \
            throw exm_error{EXM_ERR_CUDA, std::string(#call) + ": cufft error " + std::to_string((int)r_)}; \
    } while (0)

// device error word: set by kernels whose bounded waits ran out
#define EXM_DEVERR_TIMEOUT 1u
#define EXM_DEVERR_BOUNDS 2u

// ------------------------------------------------------------------ device buffers

struct exm_ctx;
struct exm_server;   // the native request loop of a context (serve.cu)

struct dbuf {
    void *p = nullptr;
    size_t bytes = 0;
};

// per-segment workspace of the analysis pipeline
struct exm_slot {
    dbuf traj;      // float2 [2][nm][nt]: (ln|z|, arg z) of H then L
    dbuf trajlo;    // float [2][nm][nt]: ln|z| - float(ln|z|), filter precision 'fp64' only (0 for uploaded trajectories)
    dbuf fft;       // double2 [2][nm][nt]: the padded rows and their transforms
    dbuf keys;      // uint32 [nm][nt]: selection scores as ordered integers
    dbuf picks;     // int32 [nm][S]: random ranks into the rest
    dbuf rej;       // int32 [1 + EXM_MAX_REJ]: rejected draw positions
    dbuf sel;       // int32 [nm][nwalk]: visited time, bit 31 set for a random draw
    dbuf hist;      // int32 histograms for the staging windows
    dbuf win;       // int32 window origins
    dbuf cnt;       // int32 [rc][48][nm+1]: taps per (lag, plane pair, template) -> offsets
    dbuf desc;      // uint4 [rc][nm*nwalk]: tap descriptors sorted by (plane pair, template)
    dbuf tside;     // int32 [rc][nm*nwalk]: time index of each descriptor (slow path)
    dbuf part;      // double [nn+1][ntau][nm]: ln of the per-lag sums
    dbuf lnl;       // double [nm]
    dbuf lnb;       // double [1]
    dbuf dev_err;   // uint32 [1]
    dbuf hostin;    // pinned host staging (d_H, d_L)
    dbuf din;       // device copy of d_H, d_L complex128 and sig2
    int nwalk = 0, rc = 0;
};

#define EXM_MAX_REJ 4096

// The last error message of a context.  The serving entry points (exm_submit, exm_poll, ...) may fail on several
// host threads at once, so an assignment is serialised, and a thread reading the message gets a copy that stays
// valid until its next read: the message of its own last failed call on this context if it has one, else the
// context's latest.  Single-threaded callers see the plain last message, as before.
struct exm_errmsg {
    exm_errmsg &operator=(const std::string &m);
    exm_errmsg &operator=(const char *m) { return *this = std::string(m); }
    operator std::string() const;   // the context's latest message (a copy)
    const char *c_str() const;      // as described above; valid until this thread's next c_str()

    exm_errmsg();

  private:
    mutable std::mutex mu_;
    std::string msg_;
    uint64_t id_;   // unique over the process's lifetime (a context made at a freed one's address gets a new id)
};

struct exm_ctx {
    int dev = 0;
    size_t budget = 0, used = 0;
    cudaStream_t stream = nullptr;
    exm_errmsg err;
    int sm_count = 148;
    size_t smem_optin = 0;

    // store (a child context borrows its parent's: it neither fills nor frees it)
    bool store_ok = false, store_borrowed = false;
    bool shard = false;         // the store is a contiguous node range of a larger store
    double s_before = 0.0;      // s of the node just below that range (0: it starts at the first node)
    exm_ctx *parent = nullptr;              // the context whose store this one borrows
    std::atomic<int> n_children{0};         // child contexts borrowing this context's store
    bool destroy_pending = false;           // destroyed while children were alive: freed with the last one
    int nn = 0, ntau = 0, nphif = 0, nb = 0, nd = 0, ndp = 0, dtype = 0;
    double beta0 = 0, dbeta = 0, delta0 = 0, ddelta = 0;
    std::vector<int64_t> tau;
    std::vector<double> s, alo, ahi;
    std::vector<char> node_set;
    dbuf T;             // [nn][ntau][nphif][nb][ndp] of float32, float16 or bfloat16 (dtype)
    size_t tstride = 0; // elements per node
    std::vector<float> tscale;   // per node: value = tscale[k] * stored element (1 for float32, bfloat16)
    dbuf d_tscale;               // float [nn]
    dbuf d_tau;         // int32 [ntau]
    CUtensorMap tmap;   // 5-D map over T for the plane windows
    bool tmap_ok = false;

    // bank (original order)
    bool bank_ok = false;
    int nm = 0, nfreq = 0, lo = 0, nt = 0;
    std::vector<float> W;
    std::vector<double> u, M, q, chi;

    // prepared analysis (internal order: templates sorted by u)
    bool prep_ok = false;
    std::vector<int> order;           // internal -> original
    std::vector<int> mlo, mhi;        // per node: valid internal template range
    std::vector<int> bnode;           // internal: boundary node or -1
    dbuf d_W;                         // float2 [nm][nfreq], internal order
    dbuf d_bhat_off;                  // double [nm]: -ln(u)/dbeta
    dbuf d_bnode;                     // int32 [nm]
    dbuf d_cb;                        // double [nm]: boundary offset (ln u + ln a_b - beta0)/dbeta
    dbuf d_lnW;                       // double [nn+1][nm]
    dbuf d_cell;                      // double [nm]
    dbuf d_mlo, d_mhi;                // int32 [nn]
    dbuf d_order;                     // int32 [nm]
    std::vector<double> ck;           // (ln s_k - beta0) / dbeta
    dbuf d_cki;                       // int32 [EXM_MAX_NODES]: floor(ck)
    dbuf d_ckd;                       // double [EXM_MAX_NODES]: ck
    dbuf d_stats;                     // uint64 [4]: gather counters (slow-path taps, boundary taps)

    // launch shape of the plane gather (index into its table; chosen by exm_autotune)
    struct exm_redshift *rs = nullptr;   // pe_redshift's grid and buffers (csrc/redshift.cu)
    int gather_cfg = 0;
    int gather_chunk_pct = 150;
    bool test_wait_expiry = false;
    bool traj_fp64 = false;          // filter precision 'fp64': the ln|z| residual is kept and used by the taps
    exm_server *srv = nullptr;       // request loop served from this context (exm_serve_start)   // the plane gather stages nothing and its barrier waits run out (a test)   // templates per gather block, percent of the one-wave-per-lag size

    // cuFFT
    cufftHandle plan = 0;
    int plan_batch = 0, plan_n = 0;
    dbuf fftwork;

    // CUDA graph of the per-segment device work (captured on first use for a shape, then replayed)
    bool use_graph = false;
    long long alloc_gen = 0;   // bumped by every allocation or free: a captured graph's buffers moved
    cudaGraphExec_t graph_exec = nullptr;
    long long graph_key[6] = {0, 0, 0, 0, 0, 0};
    double graph_node_taps = 0, graph_tlw = 0;
    long long graph_launches = 0, graph_gathers = 0;

    // CUDA-event timing of the pipeline stages on the context's stream
    bool tim_on = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pool;
    std::vector<std::pair<int, int>> ev_pending;   // (stage, pool index)
    size_t ev_used = 0;
    double tacc[8] = {0};        // ms per stage: 0 total, 1 filter, 2 select, 3 taps, 4 gather, 5 epilogue
    double node_taps = 0, tlw = 0, segments = 0;
    long long gather_launches = 0, launches = 0;

    // current segment state for the stage entry points
    exm_slot slot;
    bool traj_ok = false, times_ok = false, last_shape_ok = false;
    int cur_nwalk = 0;
    float cur_lw = 0.f;
    std::vector<exm_slot> slots;
};

// stage timers (no-ops unless timing is on): begin returns a handle for end
int exm_tim_begin(exm_ctx *ctx, int stage);
void exm_tim_end(exm_ctx *ctx, int h);
void exm_tim_collect(exm_ctx *ctx);   // after a stream synchronisation

// allocation with budget accounting
void exm_alloc(exm_ctx *ctx, dbuf &b, size_t bytes);
void exm_free(exm_ctx *ctx, dbuf &b);
void exm_ensure(exm_ctx *ctx, dbuf &b, size_t bytes);   // grow-only

// Let `func` take up to the device's opt-in shared memory per block (cudaFuncAttribute-
// MaxDynamicSharedMemorySize).  The attribute belongs to the function on the device, not to a
// context or stream, so it is raised to the largest value once per device and never lowered:
// contexts on several host threads launching the same kernel with different sizes cannot undo
// each other's setting.  Throws if `smem` exceeds the opt-in limit.
void exm_allow_smem(exm_ctx *ctx, const void *func, size_t smem);
