/*
 * exmarg_b200 -- C ABI of libexmarg_b200.so, the B200 (sm_100a) implementation of
 * exmarg's Eq. (C7) analysis path: matched filter -> table gather / log-sum-exp
 * -> distance-prior quadrature.
 *
 * Plain pointers and sizes only.  Host arrays are caller-owned and borrowed for
 * the duration of the call.  Device tables, banks and workspaces are owned by the
 * context, which enforces its HBM budget.  Every entry point returns an int
 * status (EXM_OK = 0); the message of the last failure is exm_last_error(ctx).
 * Calls on one context are serialised by the caller (one context = one stream).
 *
 * Each entry point names the reference interface it replaces (paths relative to
 * the reference repository).
 */
#ifndef EXMARG_B200_H
#define EXMARG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define EXM_API __attribute__((visibility("default")))
#else
#define EXM_API
#endif

#define EXM_OK 0
#define EXM_ERR_ARG 1     /* bad shape or argument      -> ValueError   */
#define EXM_ERR_OOM 2     /* HBM budget or allocation   -> MemoryError  */
#define EXM_ERR_CUDA 3    /* CUDA or cuFFT failure      -> RuntimeError */
#define EXM_ERR_TIMEOUT 4 /* a bounded device wait ran out -> RuntimeError */
#define EXM_ERR_STATE 5   /* call order (no store, no bank, no prepare) -> RuntimeError */

#define EXM_DTYPE_F32 0
#define EXM_DTYPE_F16 1
#define EXM_DTYPE_BF16 2

#define EXM_PRIOR_VOLUME 0
#define EXM_PRIOR_TABULATED 1 /* a density of ln y on a grid ('madau-dickinson') */
#define EXM_QUAD_GL64 16      /* OR'ed into the prior: 64-point Gauss-Legendre on every interval between
                                 a template's node points, in place of the reference's rules */

typedef struct exm_ctx exm_ctx;

/* ------------------------------------------------------------------ context */

/* Library version (major * 10000 + minor * 100 + patch). */
EXM_API int exm_version(void);

/* One analysis context on CUDA device `device` with at most `hbm_budget` bytes of
 * device memory (0: 90% of the free memory).  Replaces the implicit cupy device
 * state of exmarg/search/bank.py:17-24 (array_module) and the memory fit of
 * exmarg/search/pe.py:37-50 (_fit_chunk). */
EXM_API int exm_ctx_create(int device, size_t hbm_budget, exm_ctx **out);
EXM_API void exm_ctx_destroy(exm_ctx *ctx);

/* A second context on the parent's device that borrows the parent's resident store (its
 * tables are neither copied nor freed) and has its own stream, bank, workspace and budget:
 * several banks and segments in flight on one GPU without a second copy of the tables.
 * While children exist the parent refuses to change its store (EXM_ERR_STATE), and a
 * parent destroyed before its children keeps its tables until the last child is
 * destroyed.  No reference counterpart (one cupy device state, exmarg/search/bank.py:17-24). */
EXM_API int exm_ctx_create_sharing(exm_ctx *parent, size_t hbm_budget, exm_ctx **out);

/* enable = 1: exm_pe_intrinsic runs each segment's device work -- input copy, filter,
 * selection, taps, gather, epilogue -- as one CUDA graph, captured on the first segment
 * of a shape and replayed for the rest.  No reference counterpart. */
EXM_API int exm_ctx_set_graph(exm_ctx *ctx, int enable);

/* Scheduling priority of the context's stream (CUDA stream priorities: 0 is the default and
 * lower numbers run first; clamped to the device's range, which *range_out receives as
 * {greatest, least} if not NULL).  Contexts analysing segments at the same time compete for
 * the SMs block by block; a server that gives its workers distinct priorities lets one
 * segment's gather lead while the others fill its gaps, instead of interleaving all of them
 * (which multiplies the tap descriptors resident in L2).  No reference counterpart. */
EXM_API int exm_ctx_set_priority(exm_ctx *ctx, int priority, int *range_out);
/* The message of the last failed call on ctx.  With calls on several host threads (exm_submit and
 * exm_poll allow it), each thread gets the message of its own last failed call on ctx (else ctx's
 * latest); the pointer stays valid until the same thread calls exm_last_error again. */
EXM_API const char *exm_last_error(const exm_ctx *ctx);

/* Precision of the trajectories the table reads see.  EXM_FILTER_REFERENCE (the default): ln|z| and arg z
 * rounded once to float32, as the reference's filter leaves them (exmarg/search/bank.py:74-75); results
 * follow the reference's, float32 rounding included (at SNR 30-50 that rounding moves the reference's ln B
 * by 3e-5-7e-5 from float64).  EXM_FILTER_FP64: the float64 filter's ln|z| is kept to float64 precision (a
 * float32 residual beside the float32 value), so ln B follows float64 instead (within ~1e-5 at SNR 50); it
 * costs one more load per tap in the tap build and 4 bytes per trajectory sample.  No reference
 * counterpart. */
#define EXM_FILTER_REFERENCE 0
#define EXM_FILTER_FP64 1
EXM_API int exm_ctx_set_filter_precision(exm_ctx *ctx, int mode);

/* Test support for failure detection (no reference counterpart).  enable = 1: the plane gather of
 * this context issues no table copy, so its first bounded barrier wait runs out (after ~20k cycles
 * instead of ~1 s); the kernel then sets the device error word and returns, and the call fails with
 * EXM_ERR_TIMEOUT while the context stays usable.  No copy is in flight when a block exits.
 * enable = 0 restores normal operation. */
EXM_API int exm_ctx_test_wait_expiry(exm_ctx *ctx, int enable);
/* Bytes of device memory the context holds now. */
EXM_API size_t exm_ctx_bytes(const exm_ctx *ctx);

/* numpy's np.random.default_rng(seed).integers(0, high, count) computed on the
 * host with the same PCG64 / SeedSequence / Lemire code the selection kernel runs
 * on the device (exmarg/search/gather.py:397).  No GPU needed. */
EXM_API int exm_rng_integers(uint64_t seed, uint32_t high, int64_t count, int64_t *out);

/* Stage timing with CUDA events on the context's stream.  Returns (if out is not
 * NULL) what was accumulated since the previous call, then resets and turns timing
 * on (enable = 1) or off: out[0] device ms of whole segments (inputs already on the
 * device), out[1..5] ms of filter, selection, tap build, plane gather, epilogue,
 * out[6] plane-gather launches, out[7] node-taps, out[8] (template, lag, time)
 * taps, out[9] segments, out[10] kernel launches of this library, out[11] taps
 * that took the exact float64 path, out[12] boundary-point taps.  No reference
 * counterpart (the reference times with time.time() in its notebooks). */
EXM_API int exm_ctx_timing(exm_ctx *ctx, int enable, double *out);

/* Free and total bytes of CUDA device `device` (cudaMemGetInfo), for sizing budgets. */
EXM_API int exm_device_memory(int device, size_t *free_bytes, size_t *total_bytes);

/* ------------------------------------------------------------------ store */

/* Declare the store: n_nodes tables of shape (ntau, nphif, nb, nd), stored on the
 * device as `dtype` (EXM_DTYPE_*), lags tau_idx (ntau, in samples), the (beta,
 * Delta) grids beta0 + i dbeta and delta0 + j ddelta shared by every node.
 * Replaces exmarg/search/store.py:110-120 (upload) with resident device tables. */
EXM_API int exm_store_init(exm_ctx *ctx, int n_nodes, int ntau, int nphif, int nb, int nd, int dtype,
                   const int64_t *tau_idx, double beta0, double dbeta, double delta0, double ddelta);

/* Node k: its signal power s and amplitude-axis limits (alpha[0], alpha[-1]), and
 * its float32 table T (ntau, nphif, nb, nd, C order) copied from the host.
 * Replaces one iteration of exmarg/search/store.py:116-117 and the per-node
 * metadata of load_redshift_store (store.py:90-107). */
EXM_API int exm_store_set_node(exm_ctx *ctx, int k, double s, double alpha_lo, double alpha_hi, const float *T);

/* Nodes first .. first+n-1 loaded in one pipelined pass.  Node i's float32 table (ntau, nphif, nb, nd,
 * C order) is read from the file paths[i] at byte offset offsets[i] (the data of the uncompressed
 * T.npy member of a bd_*.npz) when paths is non-NULL and paths[i] is set, else copied from the host
 * array hosts[i].  s, alpha_lo, alpha_hi (n each, s ascending) as exm_store_set_node.
 * readers: reader threads, 1..64; chunk_bytes: staging chunk (0: 8 MiB; whole rows, at least one);
 * flags: EXM_LOAD_DIRECT reads files with O_DIRECT (no page cache) where the file system allows it
 * and with buffered reads elsewhere.  Reads fill a ring of pinned buffers while earlier chunks
 * are copied to the device; 16-bit stores are quantized on the device per node.
 * stats_out (8 doubles, may be NULL): seconds, bytes from files, bytes from host arrays, nodes
 * opened with O_DIRECT, staging buffers, chunk bytes, reader seconds (summed over threads),
 * seconds the copy issuer waited for reads.
 * Replaces load_redshift_store's table readers (exmarg/search/store.py:23-74, readers threads)
 * followed by upload (store.py:110-120). */
#define EXM_LOAD_DIRECT 1
EXM_API int exm_store_load(exm_ctx *ctx, int first, int n, const char *const *paths, const int64_t *offsets,
                           const float *const *hosts, const double *s, const double *alpha_lo, const double *alpha_hi,
                           int readers, long long chunk_bytes, int flags, double *stats_out);

/* Declare the context's store a shard: a contiguous range of the nodes of a larger store, the node
 * just below the range having signal power s_before (0 when the range starts at the first node).
 * exm_pe_prepare then sets the boundary point of the range's first node as the whole store would
 * (exmarg/search/pe.py:75-81 with s_prev = s_before) and accepts templates that reach fewer than
 * two of the shard's nodes; exm_node_values gives the whole store's rows for these nodes (and its
 * boundary row for templates whose boundary node is here, -inf elsewhere).  exm_pe_intrinsic
 * refuses a shard: the node log-sum-exp needs every shard's rows and the whole store's weights.
 * exm_store_init clears the setting.  No reference counterpart: node sharding across GPUs. */
EXM_API int exm_store_set_shard(exm_ctx *ctx, double s_before);

/* Node k filled on the device by the seeded synthetic generator (the same float32
 * values as exmarg_b200.synth.gen_table_node): T = M[b,d] * P[c] * Q[r] - S + hash
 * perturbation.  M (nb*nd), P (nphif), Q (ntau) float32.  No reference
 * counterpart: it stands in for reading bd_*.npz (store.py:23-74). */
EXM_API int exm_store_generate_node(exm_ctx *ctx, int k, double s, double alpha_lo, double alpha_hi,
                            const float *M, const float *P, const float *Q, float S, uint32_t seed);

/* Copy node k back to the host as float32 (ntau, nphif, nb, nd) (decoded for
 * 16-bit storage).  For tests. */
EXM_API int exm_store_get_node(exm_ctx *ctx, int k, float *T_out);

/* ------------------------------------------------------------------ table build */

/* Stage 2 of the offline table build (scripts/build_tables/build_k.py:59-82) on the last column and
 * last row of the (q1, q2) grid only -- all that stage 3 reads -- for every order n <= n_max:
 *   lnK_n(tau, q, phi) = float32(log(max(K_n, 1e-300)) + gmo[n]),
 *   K_n = sum_m cosm[m][phi] sum_{a - b = m} coeff[key] Wd[key][tau] exp((a+b) lq1 + (2n-a-b) lq2 - 2n lq_last)
 * with (lq1, lq2) = (lnq[q], lnq[nq-1]) for the column and (lnq[nq-1], lnq[q]) for the row.
 * Wd (n_keys, n_tau): the node's W rebinned onto the data delays, keys (n, a, b <= a) in order;
 * coeff (n_keys): C(n,a) C(n,b) (2 when a > b); gmo (n_max+1): 2n lnq[nq-1] - ln(n! s^n);
 * cosm (n_max+1, nphif): cos(m phi_p).  col_out, row_out: float32 (n_max+1, n_tau, nq, nphif), the
 * inputs of exm_bd_build.  ms_out (may be NULL): kernel milliseconds.  No 49 GB lnK is formed. */
EXM_API int exm_k_edges(exm_ctx *ctx, int n_max, int n_tau, const double *Wd, const double *coeff, int nq,
                        const double *lnq, const double *gmo, int nphif, const double *cosm, float *col_out,
                        float *row_out, double *ms_out);

/* Stage 3 of the offline table build (scripts/build_tables/build_bd.py:53-77): one node's table
 * T[tau, phi, beta, Delta] = log sum_{n <= n_max} exp(n beta + g_n(Delta)), float64 arithmetic,
 * float32 result, for each truncation order n_max in ladder (n_ladder of them).
 * col, row: float32 (nord, ntau, nq, nphif), the last column lnK[n, tau, :, nq-1, :nphif] and the
 * last row lnK[n, tau, nq-1, :, :nphif] of stage 2's lnK (nord orders, nq magnitudes);
 * lnq (nq) the log magnitudes, beta (nb) the beta grid.  T_out: n_ladder tables of
 * (ntau, nphif, nb, 2 nq - 1) float32, Delta ascending as build_bd.py:57 orders it.
 * n_nonfinite_out: entries that are not finite (the reference then refuses the table);
 * ms_out (may be NULL): kernel milliseconds, milliseconds including the copies. */
EXM_API int exm_bd_build(exm_ctx *ctx, int nord, int ntau, int nq, int nphif, const float *col, const float *row,
                         const double *lnq, int nb, const double *beta, int n_ladder, const int *ladder,
                         float *T_out, long long *n_nonfinite_out, double *ms_out);

/* Stage 1 of the offline table build (scripts/build_tables/w_gpu.py:67-182): the GORFs at fixed
 * distance W_j(tau, key) at n_nodes nodes s_nodes, keys (n, a, b), b <= a <= n <= n_max, in the order
 * n, a, b ascending, by quadrature over n_pix sky pixels and the (psi, chi) grid, float64, result
 * float32 (n_nodes, n_tau, n_keys) in W_out.
 * c2p, s2p (n_psi) float32 cos 2psi, sin 2psi; ap, cg (n_chi) float32 (1 + chi^2)/2 and chi;
 * wq (n_chi) float64 quadrature weights; resp (n_pix, 4) float32 F+_H, Fx_H, F+_L, Fx_L at psi = 0;
 * j0 (n_pix) the lower delay bin of each pixel, w (n_pix, 2) its deposit weights on bins j0, j0 + 1;
 * scale (n_nodes, n_keys) the per-(node, order) factor s^n 2^n / n!.
 * n_nonfinite_out: entries that are not finite; ms_out (may be NULL): quadrature milliseconds,
 * milliseconds in all.  Replaces w_table_s_gpu (w_gpu.py:134-182) with one pixel per step. */
EXM_API int exm_w_build(exm_ctx *ctx, int n_nodes, const double *s_nodes, int n_max, int n_psi, int n_chi,
                        const float *c2p, const float *s2p, const float *ap, const float *cg, const double *wq,
                        int n_pix, const float *resp, const int *j0, const double *w, int n_tau, const double *scale,
                        float *W_out, long long *n_nonfinite_out, double *ms_out);

/* ------------------------------------------------------------------ bank */

/* The template bank: nm templates of nfreq complex64 factors W = a e^{i psi0}
 * (interleaved re, im), starting at frequency bin `lo` of a grid whose filter
 * length is n_time = 8 nu_max; u (nm) the template powers; M, q, chi (nm) the
 * bank axes (for the cell weights of ln B).  Replaces the device copy of
 * exmarg/search/bank.py:35-54 (MassBank.__init__). */
EXM_API int exm_bank_set(exm_ctx *ctx, int nm, int nfreq, int lo, int n_time, const float *W, const double *u,
                 const double *M, const double *q, const double *chi);

/* ------------------------------------------------------------------ analysis */

/* Node geometry (exmarg/search/pe.py:58-84), distance-prior weights
 * (pe.py:260-286 and :321-327, computed on the device in float64) and cell
 * weights (pe.py:338-343) for the current store and bank.  prior
 * EXM_PRIOR_VOLUME, or EXM_PRIOR_TABULATED with the density (lny, p_lny) of
 * n_dens points ('madau-dickinson', exmarg/priors.py:31-38); | EXM_QUAD_GL64
 * integrates every interval with 64 Gauss-Legendre points in ln y instead of the
 * reference's closed form (volume) or 401-point trapezoid (tabulated).  Fails with
 * EXM_ERR_ARG and the reference's message when a template reaches fewer than
 * two nodes (pe.py:324-325). */
EXM_API int exm_pe_prepare(exm_ctx *ctx, double ymin, int prior, const double *lny, const double *p_lny, int n_dens);

/* The n-point Gauss-Legendre rule on [-1, 1] (n <= 256), nodes x (ascending) and weights w, float64, by Newton
 * iteration on the Legendre recurrence: the rule exm_pe_prepare uses with EXM_QUAD_GL64 (64 points).  No GPU
 * needed.  No reference counterpart (the reference integrates in closed form or by the trapezoid rule,
 * exmarg/search/pe.py:260-286). */
EXM_API int exm_gauss_legendre(int n, double *x, double *w);

/* pe_intrinsic on n_seg segments (exmarg/search/pe.py:289-346): d_H, d_L
 * (n_seg, nfreq) complex128 (interleaved), sig2_H, sig2_L (nfreq) float64,
 * seeds (n_seg) the random-draw seed of each segment (seed + row),
 * n_loud / n_random as gather.select_times (n_loud = 0: every arrival time).
 * Outputs ln_lambda (n_seg, nm) and ln_b (n_seg) float64 on the host. */
EXM_API int exm_pe_intrinsic(exm_ctx *ctx, int n_seg, const double *d_H, const double *d_L, const double *sig2_H,
                     const double *sig2_L, const int64_t *seeds, int n_loud, int n_random, double *ln_lambda,
                     double *ln_b);

/* Autotuner of the plane gather's launch shape (warps per block x taps per register
 * group): replays the gather of the last segment analysed by exm_pe_intrinsic on this
 * context (same n_loud, n_random) once per shape, times each with CUDA events (reps
 * launches), keeps the fastest for later calls and writes its index to best_cfg and the
 * ms per launch of every shape to ms_per_cfg (if not NULL; room for 16 entries: this build
 * has 5 shapes, warps per block including the producer warp x taps per register group:
 * 28x1 (an untuned context's), 16x2, 24x2, 24x1, 20x2).  Then, with the best shape, it times
 * the templates per gather block at 50, 150 and 200 percent of one wave of blocks per lag
 * (measured at 100) into ms_per_cfg[5..7], and keeps the best percentage (best_chunk_pct, if
 * not NULL; an untuned context uses 150).
 * No reference counterpart (the reference takes block as a kwarg, pe.py:289-290). */
EXM_API int exm_autotune(exm_ctx *ctx, int n_loud, int n_random, int reps, int *best_cfg, int *best_chunk_pct,
                         double *ms_per_cfg);

/* Select a launch shape of the plane gather by index (as exm_autotune reports it) and the
 * templates per gather block in percent of one wave of blocks per lag (10..1000; 0 keeps the
 * current; an untuned context uses shape 0 at 150). */
EXM_API int exm_set_gather_cfg(exm_ctx *ctx, int cfg, int chunk_pct);

/* ------------------------------------------------------------------ serving (native request loop) */

/* Start a request loop on ctx, the context that owns the resident store.  The reference analyses one
 * pe_intrinsic call at a time (exmarg/search/pe.py:289-346); this loop admits requests continuously:
 * workers are child contexts (exm_ctx_create_sharing) on host threads of their own, each holding one
 * bank and one workspace, opened and closed within hbm_budget bytes (0: 85% of the free device memory)
 * and max_workers (1..64).  A request starts on an idle worker of its bank; a bank with no worker may
 * close idle workers of banks with nothing queued to make room; a bank whose workers are busy waits for
 * one unless the budget has room for another.  A worker's cost is estimated from its bank's shape until
 * its first segment has run, then measured.  Every request uses n_loud / n_random (as exm_pe_intrinsic)
 * and, with use_graph, each worker replays its segments as a captured CUDA graph.  Workers take ctx's
 * gather launch shape, so a served result is bitwise exm_pe_intrinsic's on ctx for the same bank,
 * segment and seed, whatever runs beside it.  Requests started while others run get decreasing stream
 * priorities (the oldest leads). */
EXM_API int exm_serve_start(exm_ctx *ctx, size_t hbm_budget, int max_workers, int n_loud, int n_random,
                            int use_graph);

/* Register a bank with the server (before the first request): as exm_bank_set (nm <= 8192) followed
 * by exm_pe_prepare (ymin, prior, density).  *bank_id receives its id for exm_submit.  Replaces
 * mass_bank's device state (exmarg/search/bank.py:35-54) held per worker. */
EXM_API int exm_serve_add_bank(exm_ctx *ctx, int nm, int nfreq, int lo, int n_time, const float *W,
                               const double *u, const double *M, const double *q, const double *chi, double ymin,
                               int prior, const double *lny, const double *p_lny, int n_dens, int *bank_id);

/* Queue one segment for bank bank_id and return at once with *handle.  d_H, d_L: (nfreq) complex128
 * (interleaved), sig2_H, sig2_L: (nfreq) float64 -- copied, so the caller's buffers are free when this
 * returns; seed: the random-draw seed of the segment (the reference's seed + row).  The equivalent of
 * one row of pe_intrinsic (exmarg/search/pe.py:289-346).  Safe to call from several host threads. */
EXM_API int exm_submit(exm_ctx *ctx, int bank_id, const double *d_H, const double *d_L, const double *sig2_H,
                       const double *sig2_L, int64_t seed, int64_t *handle);

/* Wait up to timeout_us microseconds (0: do not wait; negative: until done) for request `handle`.
 * EXM_OK: ln_lambda (the bank's nm, float64, bank order) and *ln_b are written and the handle is
 * released; EXM_ERR_TIMEOUT: not finished yet (poll again); any other status: the request failed
 * (message in exm_last_error) and the handle is released.  Safe to call from several host threads. */
EXM_API int exm_poll(exm_ctx *ctx, int64_t handle, int64_t timeout_us, double *ln_lambda, double *ln_b);

/* An idle worker is closed to make room for another bank only after it has been idle for `seconds` (default
 * 0.25; 0: at once).  With a mix of banks whose workers do not fit the budget together, closing at once turns
 * every bank change into a close and an open (seconds each); the minimum idle time bounds that churn, and the
 * request of a bank without a worker waits for a worker to qualify.  No reference counterpart. */
EXM_API int exm_serve_set_min_idle(exm_ctx *ctx, double seconds);

/* Server counters, out (10 doubles): requests served, failed, queued, running; workers open, opened in
 * all, closed for budget; workspace bytes in use (estimated or measured), the budget; seconds from the
 * first request of an idle server to the last result. */
EXM_API int exm_serve_stats(exm_ctx *ctx, double *out);

/* Stop the server: running requests finish, queued ones fail, workers close; handles not yet polled
 * become invalid.  exm_ctx_destroy stops a server that is still running. */
EXM_API int exm_serve_stop(exm_ctx *ctx);

/* ------------------------------------------------------------------ stages (tests, gather-level drop-in) */

/* Matched filter of one segment (exmarg/search/bank.py:56-78, MassBank.trajectories):
 * the result stays on the device for the next stages; traj_out, if not NULL,
 * receives float32 (4, nm, n_time) = lqH, phH, lqL, phL. */
EXM_API int exm_filter(exm_ctx *ctx, const double *d_H, const double *d_L, const double *sig2_H, const double *sig2_L,
               float *traj_out);

/* Upload trajectories (4, nm, n_time) float32 = lqH, phH, lqL, phL from the host,
 * in place of exm_filter. */
EXM_API int exm_set_trajectories(exm_ctx *ctx, const float *traj);

/* Time selection of the current trajectories (exmarg/search/gather.py:374-420,
 * select_times), with the numpy PCG64 draw of np.random.default_rng(seed)
 * reproduced on the device.  sel_out (nm, n_loud + n_random) int32 and lw_out
 * float32, if not NULL, receive the result. */
EXM_API int exm_select_times(exm_ctx *ctx, int64_t seed, int n_loud, int n_random, int32_t *sel_out, float *lw_out);

/* The float32 exp the selection scores use, on the device: y[i] = exp(x[i]) for n host values,
 * bit for bit numpy's float32 np.exp (its SIMD kernel on AVX2 / AVX-512 hosts), the exp of the
 * reference's score (exmarg/search/gather.py:407).  For tests of the selection's arithmetic. */
EXM_API int exm_np_exp32(exm_ctx *ctx, const float *x, float *y, int64_t n);

/* Upload a time selection (nm, nwalk) from the host in place of exm_select_times
 * (nwalk = 0: every arrival time). */
EXM_API int exm_set_times(exm_ctx *ctx, int nwalk, const int32_t *sel, const float *lw);

/* The gather contract of exmarg/search/gather.py:114-140 / :340-371
 * (gather_cpu / gather_gpu) on the current trajectories and times: nsel
 * (template, slot) rows, mass_ids (nsel), lna and tab_ids (nsel, ns); out
 * (ns, nsel) float64 ln Lambda.  Arithmetic in float64 like the reference CPU
 * path. */
EXM_API int exm_gather(exm_ctx *ctx, int nsel, int ns, const int64_t *mass_ids, const double *lna, const int64_t *tab_ids,
               double *out);

/* The float64 gather of exm_gather for callers that cannot allocate device memory
 * during the call (a framework whose memory pool owns the device, a spent budget, a
 * context where an allocation would synchronise).  No counterpart in the reference.
 * Every argument is a device pointer the caller owns: lqH, phH, lqL, phL (nm, n_time)
 * float32 trajectories; sel, lw (nm, nwalk) visited times and their log weights
 * (nwalk = 0: every time); mass_ids (nsel) int64, lna (nsel, ns) float64, tab_ids
 * (nsel, ns) int64 node indices into the context's resident store; out (ns, nsel)
 * float64.  The call allocates nothing: its partial sums live in a fixed device array
 * of the library (16 MiB, held by every device that loads the library), so
 * ns * n_lag * nsel must not exceed 2^20 (larger requests fail with EXM_ERR_ARG).
 * exm_ctx_create loads the array and this call's kernels on its device and looks the
 * array's device address up (cudaGetSymbolAddress), so no call allocates, the first
 * included; the address is refreshed by every context creation and assumes the device's
 * primary context outlives the contexts.  Calls share the array and its error word: do
 * not run two calls at once on one device (two contexts or streams); they would race.
 * Out-of-range mass ids, table ids or visited times fail with EXM_ERR_ARG.  It runs on
 * the context's stream and returns after the result is written. */
EXM_API int exm_gather_noalloc(exm_ctx *ctx, int nm, int n_time, const float *lqH, const float *phH,
                               const float *lqL, const float *phL, int nwalk, const int32_t *sel, const float *lw,
                               int nsel, int ns, const int64_t *mass_ids, const double *lna, const int64_t *tab_ids,
                               double *out);

/* pe_redshift's grid (exmarg/search/pe.py:203-257): the node geometry's y values yN
 * (nn1 = n_nodes + 1 rows, row n_nodes the boundary point, nm templates in bank order), the
 * bank's detector-frame total masses Mdet (ascending), the z grid and yq = D0 / D_L(z) (nz),
 * the source-frame primary masses m1 (nm1) and the normalised prior weights w (nm1, nz).
 * Kept on the device for exm_source_frame; replaces a previous grid.  No counterpart in the
 * reference as a separate call (it is part of its pe_redshift). */
EXM_API int exm_redshift_grid(exm_ctx *ctx, int nn1, int nm, const double *yN, const double *Mdet, int nz,
                      const double *yq, const double *z, int nm1, const double *m1, const double *w);

/* One segment's source frame (exmarg/search/pe.py:87-132, _to_source_frame, and the ln B of
 * :249-255): node values lamN (nn1, nm, as exm_node_values gives them) -> ln_lambda_out
 * (nm1, nz; may be NULL) and ln_b_out, float64, on the grid of exm_redshift_grid. */
EXM_API int exm_source_frame(exm_ctx *ctx, const double *lamN, double *ln_lambda_out, double *ln_b_out);

/* Node values of the current segment (exmarg/search/pe.py:168-200,
 * _node_values): lamN_out (n_nodes + 1, nm) float64, -inf where a template does
 * not reach a node; row n_nodes the boundary point.  Uses the plane-staged gather. */
EXM_API int exm_node_values(exm_ctx *ctx, double *lamN_out);

#ifdef __cplusplus
}
#endif

#endif
