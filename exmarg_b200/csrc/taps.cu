// Tap descriptors for the plane-staged gather.
//
// A tap is one (template, walked time, lag).  Its plane pair p, the weight of plane
// p + 1, beta-hat and the Delta coordinate do not depend on the node, so they are
// computed once per tap (in float64, as the reference computes them per node) and
// packed into 16 bytes:
//   x = fb (float, fraction of beta-hat), y = fd (float, fraction of Delta),
//   z = w (float, weight of plane p + 1) | bit 31: the time is a random draw,
//   w = template (13 bits) << 19 | rd (8 bits) << 11 | rb0 (11 bits, signed),
// with the staging windows already placed (k_windows runs between the count and the
// scatter): rd = d0 - C0, the column inside every node's window (255: outside, the
// exact path), and rb0 = floor(beta-hat) - Rh, the row relative to the window row
// origin in beta-hat; node k's window row of the tap is then rb0 + carry + a constant
// of the node, so the gather adds only the node's part.
// For each lag the descriptors are counting-sorted by (p, template), so every node's
// gather block reads, for each plane pair it has staged, one contiguous run per warp.
// A second array holds each descriptor's time index for the exact slow path.
#include "common.cuh"
#include "kernels.cuh"

struct TapArgs {
    const float2 *H, *L;
    const float *Hlo, *Llo;   // residuals of ln|z| (filter precision 'fp64'), else null
    const int32_t *sel;
    const double *boff;   // [nmc] -ln(u)/dbeta of the chunk's templates
    const int *tau;       // [ntau]
    int *cnt;             // [rc][48][nmc + 1]
    int *hist_b;          // [EXM_HB_N]
    int *hist_d;          // [256]
    uint4 *desc;
    int32_t *tside;
    TapGeom g;
    int nmc, nwalk, use_sel, r0, want_hb;
    long long per_lag;    // nmc * nwalk
    long long pitch;      // descriptors stored per lag (whole chunks, exm_desc_pitch)
    const int *win;       // window origins (k_windows): [0] column C0, [1 + EXM_MAX_NODES] beta-hat row Rh
    int wd;               // window columns
};

__device__ __forceinline__ void tap_time(const TapArgs &a, int i, int k, int &t, int &flag)
{
    if (a.use_sel) {
        const int v = a.sel[(long long)i * a.nwalk + k];
        t = v & 0x7FFFFFFF;
        flag = (unsigned)v >> 31;
    } else {
        t = k;
        flag = 0;
    }
}

#define TAP_CACHE 4096   // walked times of one template cached in shared memory (time, L sample)

// the walked times of template i and their L samples, in shared memory when they fit
struct WalkCache {
    int *t;        // the time, bit 31: a random draw
    float2 *l;
    float *llo;
    bool on;
};

__device__ __forceinline__ void load_walk(const TapArgs &a, int i, const float2 *L, const float *Llo, WalkCache &wc)
{
    if (!wc.on) return;
    for (int k = threadIdx.x; k < a.nwalk; k += blockDim.x) {
        int t, flag;
        tap_time(a, i, k, t, flag);
        wc.t[k] = (int)((unsigned)t | ((unsigned)flag << 31));
        wc.l[k] = L[t];
        wc.llo[k] = Llo ? Llo[t] : 0.f;
    }
    __syncthreads();
}

__device__ __forceinline__ void walk_at(const TapArgs &a, int i, const float2 *L, const float *Llo, const WalkCache &wc,
                                        int k, int &t, int &flag, float2 &l, float &llo)
{
    if (wc.on) {
        const int v = wc.t[k];
        t = v & 0x7FFFFFFF;
        flag = (unsigned)v >> 31;
        l = wc.l[k];
        llo = wc.llo[k];
    } else {
        tap_time(a, i, k, t, flag);
        l = L[t];
        llo = Llo ? Llo[t] : 0.f;
    }
}

// counts per (lag, pair, template), and the histograms that place the staging windows: one
// block per template walks every lag of the chunk; the histograms are flushed once per block
__global__ void __launch_bounds__(256) k_tap_count(TapArgs a, int rc)
{
    __shared__ int c[EXM_NPAIR];
    __shared__ int hd[256];
    __shared__ int hb[EXM_HB_N];
    extern __shared__ unsigned char wsm[];
    const int i = blockIdx.x;
    const bool do_hb = a.want_hb;
    for (int q = threadIdx.x; q < 256; q += blockDim.x) hd[q] = 0;
    if (do_hb)
        for (int q = threadIdx.x; q < EXM_HB_N; q += blockDim.x) hb[q] = 0;
    const int nt = a.g.nt;
    const float2 *H = a.H + (long long)i * nt, *L = a.L + (long long)i * nt;
    const float *Hlo = a.Hlo ? a.Hlo + (long long)i * nt : nullptr, *Llo = a.Llo ? a.Llo + (long long)i * nt : nullptr;
    const double boff = a.boff[i];
    WalkCache wc;
    wc.on = a.nwalk <= TAP_CACHE;
    wc.l = (float2 *)wsm;
    wc.t = (int *)(wc.l + TAP_CACHE);
    wc.llo = (float *)(wc.t + TAP_CACHE);
    load_walk(a, i, L, Llo, wc);
    for (int rl = 0; rl < rc; ++rl) {
        for (int q = threadIdx.x; q < EXM_NPAIR; q += blockDim.x) c[q] = 0;
        __syncthreads();
        const int tau0 = ((a.tau[a.r0 + rl] % nt) + nt) % nt;
        for (int k = threadIdx.x; k < a.nwalk; k += blockDim.x) {
            int t, flag;
            float2 l;
            float llo;
            walk_at(a, i, L, Llo, wc, k, t, flag, l, llo);
            int i1 = t + tau0;
            if (i1 >= nt) i1 -= nt;
            int p, ib, d0;
            float w, fb, fd;
            exm_tap_geom(l, H[i1], llo, Hlo ? Hlo[i1] : 0.f, boff, a.g, p, w, ib, fb, d0, fd);
            // warp-aggregated increments: one atomic per distinct bin in the warp
            const unsigned pm = __match_any_sync(__activemask(), p);
            if ((threadIdx.x & 31) == __ffs(pm) - 1) atomicAdd(&c[p], __popc(pm));
            const unsigned dm = __match_any_sync(__activemask(), d0);
            if ((threadIdx.x & 31) == __ffs(dm) - 1) atomicAdd(&hd[d0], __popc(dm));
            if (do_hb && rl == 0) atomicAdd(&hb[ib - EXM_HB_LO], 1);
        }
        __syncthreads();
        for (int q = threadIdx.x; q < EXM_NPAIR; q += blockDim.x)
            a.cnt[((long long)rl * EXM_NPAIR + q) * (a.nmc + 1) + i] = c[q];
    }
    __syncthreads();
    for (int q = threadIdx.x; q < 256; q += blockDim.x)
        if (hd[q]) atomicAdd(&a.hist_d[q], hd[q]);
    if (do_hb)
        for (int q = threadIdx.x; q < EXM_HB_N; q += blockDim.x)
            if (hb[q]) atomicAdd(&a.hist_b[q], hb[q]);
}

// exclusive scan over (pair, template) per lag: cnt becomes the start offsets; column
// nmc of pair p is the start of pair p + 1
__global__ void __launch_bounds__(1024) k_tap_scan(int *cnt, int nmc)
{
    __shared__ int sh[33];
    const int rl = blockIdx.x;
    int *c = cnt + (long long)rl * EXM_NPAIR * (nmc + 1);
    const int n = EXM_NPAIR * nmc;
    int carry = 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < n; base += blockDim.x) {
        const int e = base + threadIdx.x;
        const int p = e / nmc, i = e - p * nmc;
        const int v = (e < n) ? c[p * (nmc + 1) + i] : 0;
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) sh[warp] = x;
        __syncthreads();
        if (warp == 0) {
            int s = sh[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += y;
            }
            sh[lane] = s;
        }
        __syncthreads();
        const int excl = carry + x - v + (warp ? sh[warp - 1] : 0);
        if (e < n) c[p * (nmc + 1) + i] = excl;
        const int tot = sh[31];
        __syncthreads();
        carry += tot;
    }
    __syncthreads();
    for (int p = threadIdx.x; p < EXM_NPAIR; p += blockDim.x)
        c[p * (nmc + 1) + nmc] = (p + 1 < EXM_NPAIR) ? c[(p + 1) * (nmc + 1)] : carry;
}

// descriptors, stably scattered to their (lag, pair, template) runs: one block per template,
// every lag of the chunk in turn.  A batch is SCATTER_ROUNDS rounds of 256 walked times (k = k0 + m 256 +
// thread): each warp counts its taps per pair in each round, 48 threads turn the counts into exclusive
// prefixes in (round, warp) order -- the order of k -- and every tap lands at its run's base + the prefix + its
// rank among equal pairs in the warp: the same positions as one walked time per thread and round, with four
// block barriers per batch instead of four per round.
#define SCATTER_ROUNDS 4
__global__ void __launch_bounds__(256) k_tap_scatter(TapArgs a, int rc)
{
    __shared__ int wcnt[SCATTER_ROUNDS][8][EXM_NPAIR];
    __shared__ int base[EXM_NPAIR];
    extern __shared__ unsigned char wsm[];
    const int i = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nt = a.g.nt;
    const float2 *H = a.H + (long long)i * nt, *L = a.L + (long long)i * nt;
    const float *Hlo = a.Hlo ? a.Hlo + (long long)i * nt : nullptr, *Llo = a.Llo ? a.Llo + (long long)i * nt : nullptr;
    const double boff = a.boff[i];
    WalkCache wc;
    wc.on = a.nwalk <= TAP_CACHE;
    wc.l = (float2 *)wsm;
    wc.t = (int *)(wc.l + TAP_CACHE);
    wc.llo = (float *)(wc.t + TAP_CACHE);
    load_walk(a, i, L, Llo, wc);
    const unsigned lt = (1u << lane) - 1u;
    const int C0 = a.win[0], Rh = a.win[1 + EXM_MAX_NODES];
    for (int rl = 0; rl < rc; ++rl) {
        const int tau0 = ((a.tau[a.r0 + rl] % nt) + nt) % nt;
        const int *off = a.cnt + (long long)rl * EXM_NPAIR * (a.nmc + 1);
        uint4 *desc = a.desc + (long long)rl * a.pitch;
        int32_t *tside = a.tside + (long long)rl * a.pitch;
        __syncthreads();
        for (int q = threadIdx.x; q < EXM_NPAIR; q += blockDim.x) base[q] = off[q * (a.nmc + 1) + i];
        for (int k0 = 0; k0 < a.nwalk; k0 += SCATTER_ROUNDS * 256) {
            for (int q = threadIdx.x; q < SCATTER_ROUNDS * 8 * EXM_NPAIR; q += blockDim.x) (&wcnt[0][0][0])[q] = 0;
            __syncthreads();
            int p[SCATTER_ROUNDS], rk[SCATTER_ROUNDS], tt[SCATTER_ROUNDS];
            uint4 d[SCATTER_ROUNDS];
#pragma unroll
            for (int m = 0; m < SCATTER_ROUNDS; ++m) {
                const int k = k0 + m * 256 + threadIdx.x;
                int t = 0, flag = 0, ib = 0, d0 = 0;
                float w = 0.f, fb = 0.f, fd = 0.f;
                p[m] = -1;
                if (k < a.nwalk) {
                    float2 l;
                    float llo;
                    walk_at(a, i, L, Llo, wc, k, t, flag, l, llo);
                    int i1 = t + tau0;
                    if (i1 >= nt) i1 -= nt;
                    exm_tap_geom(l, H[i1], llo, Hlo ? Hlo[i1] : 0.f, boff, a.g, p[m], w, ib, fb, d0, fd);
                }
                const unsigned peers = __match_any_sync(0xffffffffu, p[m]);
                rk[m] = __popc(peers & lt);
                if (p[m] >= 0 && rk[m] == 0) wcnt[m][warp][p[m]] = __popc(peers);
                d[m].x = __float_as_uint(fb);
                d[m].y = __float_as_uint(fd);
                d[m].z = __float_as_uint(w) | ((unsigned)flag << 31);
                int rd = d0 - C0, rb0 = ib - Rh;
                if ((unsigned)rd > (unsigned)(a.wd - 2) || rb0 < -1024 || rb0 > 1023) {
                    rd = 255;   // outside every node's window: the exact path
                    rb0 = 0;
                }
                d[m].w = ((unsigned)i << 19) | ((unsigned)rd << 11) | ((unsigned)rb0 & 0x7FFu);
                tt[m] = t;
            }
            __syncthreads();
            if (threadIdx.x < EXM_NPAIR) {   // exclusive prefixes per pair in (round, warp) order, from the run base
                const int q = threadIdx.x;
                int run = base[q];
                for (int m = 0; m < SCATTER_ROUNDS; ++m)
                    for (int ww = 0; ww < 8; ++ww) {
                        const int v = wcnt[m][ww][q];
                        wcnt[m][ww][q] = run;
                        run += v;
                    }
                base[q] = run;
            }
            __syncthreads();
#pragma unroll
            for (int m = 0; m < SCATTER_ROUNDS; ++m) {
                if (p[m] < 0) continue;
                const int pos = wcnt[m][warp][p[m]] + rk[m];
                if (pos >= 0 && pos < a.per_lag) {
                    desc[pos] = d[m];   // sorted order; k_tap_interleave rearranges each chunk afterwards
                    tside[pos] = tt[m];
                }
            }
            __syncthreads();
        }
    }
}

// Each chunk of EXM_DCH descriptors (and time indices) of every lag, from sorted order to the
// gather's lane-interleaved order (exm_desc_phys), in place through shared memory: writing the
// interleaved order directly from the scatter would spread 16-byte stores over many sectors.
__global__ void __launch_bounds__(256) k_tap_interleave(uint4 *__restrict__ desc, int32_t *__restrict__ tside,
                                                        long long n_chunks)
{
    __shared__ uint4 sd[EXM_DCH];
    __shared__ int32_t st[EXM_DCH];
    for (long long ch = blockIdx.x; ch < n_chunks; ch += gridDim.x) {
        uint4 *d = desc + ch * EXM_DCH;
        int32_t *t = tside + ch * EXM_DCH;
        for (int q = threadIdx.x; q < EXM_DCH; q += blockDim.x) {
            sd[q] = d[q];
            st[q] = t[q];
        }
        __syncthreads();
        // storage index i*32 + l holds sorted position l*TPL + i
        for (int ph = threadIdx.x; ph < EXM_DCH; ph += blockDim.x) {
            const int q = (ph & 31) * EXM_TPL + (ph >> 5);
            d[ph] = sd[q];
            t[ph] = st[q];
        }
        __syncthreads();
    }
}

// staging-window origins: column C0 (a multiple of calign elements, 16 bytes), per node the
// first beta row, and the beta-hat row origin Rh they derive from; wd columns per window
__global__ void k_windows(const int *hist_b, const int *hist_d, const int *cki, int nn, int nb, int nd, int ndp,
                          int wd, int calign, int *win)
{
    __shared__ long long best[2];
    if (threadIdx.x == 0) best[0] = best[1] = 0;
    __syncthreads();
    // columns: d0 in [C0, C0 + wd - 2]
    const int cmax = max(0, ndp - wd);
    for (int c0 = threadIdx.x * calign; c0 <= cmax; c0 += blockDim.x * calign) {
        long long s = 0;
        for (int d = c0; d <= min(c0 + wd - 2, nd - 1); ++d) s += hist_d[d];
        long long key = (s << 12) | (4095 - c0 / calign);
        atomicMax((unsigned long long *)&best[0], (unsigned long long)key);
    }
    // beta-hat rows: ib in [Rh, Rh + WB - 3]
    for (int rh = threadIdx.x; rh < EXM_HB_N; rh += blockDim.x) {
        long long s = 0;
        for (int x = rh; x <= min(rh + EXM_WB - 3, EXM_HB_N - 1); ++x) s += hist_b[x];
        long long key = (s << 12) | (4095 - rh);
        atomicMax((unsigned long long *)&best[1], (unsigned long long)key);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        win[0] = (4095 - (int)(best[0] & 4095)) * calign;
        const int rh = (4095 - (int)(best[1] & 4095)) + EXM_HB_LO;
        for (int k = 0; k < nn; ++k) {
            int r0 = rh + cki[k];
            r0 = max(0, min(r0, nb - EXM_WB));
            win[1 + k] = r0;
        }
        win[1 + EXM_MAX_NODES] = rh;
    }
}

void exm_run_taps(exm_ctx *ctx, exm_slot &sl, const ChunkInfo &ci, int r0, int rc, bool first_chunk_of_lags)
{
    const int nt = ctx->nt;
    TapArgs a;
    a.H = (const float2 *)sl.traj.p;
    a.L = a.H + (size_t)ci.nmc * nt;
    a.Hlo = ctx->traj_fp64 ? (const float *)sl.trajlo.p : nullptr;
    a.Llo = a.Hlo ? a.Hlo + (size_t)ci.nmc * nt : nullptr;
    a.sel = (const int32_t *)sl.sel.p;
    a.boff = (const double *)ctx->d_bhat_off.p + ci.m_base;
    a.tau = (const int *)ctx->d_tau.p;
    a.cnt = (int *)sl.cnt.p;
    a.hist_b = (int *)sl.hist.p;
    a.hist_d = a.hist_b + EXM_HB_N;
    a.desc = (uint4 *)sl.desc.p;
    a.tside = (int32_t *)sl.tside.p;
    a.g.rph = EXM_NPHI / 6.283185307179586;
    a.g.rdb = 2.0 / ctx->dbeta;
    a.g.rdd = 1.0 / ctx->ddelta;
    a.g.offd = -ctx->delta0 / ctx->ddelta;
    a.g.nd = ctx->nd;
    a.g.nt = nt;
    a.nmc = ci.nmc;
    a.nwalk = ci.nwalk;
    a.use_sel = ci.use_sel;
    a.r0 = r0;
    a.want_hb = first_chunk_of_lags ? 1 : 0;
    a.per_lag = (long long)ci.nmc * ci.nwalk;
    a.pitch = exm_desc_pitch(a.per_lag);
    if (first_chunk_of_lags) EXM_CUDA(cudaMemsetAsync(a.hist_b, 0, sizeof(int) * EXM_HB_N, ctx->stream));
    EXM_CUDA(cudaMemsetAsync(a.hist_d, 0, sizeof(int) * 256, ctx->stream));
    const size_t wsm = a.nwalk <= TAP_CACHE ? (size_t)TAP_CACHE * (sizeof(float2) + sizeof(int) + sizeof(float)) : 0;
    exm_allow_smem(ctx, (const void *)k_tap_count, wsm);
    exm_allow_smem(ctx, (const void *)k_tap_scatter, wsm);
    a.win = (const int *)sl.win.p;
    a.wd = exm_dtype_wd(ctx->dtype);
    k_tap_count<<<ci.nmc, 256, wsm, ctx->stream>>>(a, rc);
    k_tap_scan<<<rc, 1024, 0, ctx->stream>>>(a.cnt, ci.nmc);
    k_windows<<<1, 256, 0, ctx->stream>>>(a.hist_b, a.hist_d, (const int *)ctx->d_cki.p, ctx->nn, ctx->nb, ctx->nd, ctx->ndp,
                                          exm_dtype_wd(ctx->dtype), exm_dtype_calign(ctx->dtype), (int *)sl.win.p);
    k_tap_scatter<<<ci.nmc, 256, wsm, ctx->stream>>>(a, rc);
    const long long n_chunks = (long long)rc * a.pitch / EXM_DCH;
    k_tap_interleave<<<(int)std::min<long long>(n_chunks, (long long)ctx->sm_count * 32), 256, 0, ctx->stream>>>(
        a.desc, a.tside, n_chunks);
    EXM_CUDA(cudaGetLastError());
    ctx->launches += 5;
}
