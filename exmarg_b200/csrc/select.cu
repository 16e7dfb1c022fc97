// Time selection of one segment (exmarg/search/gather.py:374-420, select_times):
//   score(t) = exp(2 ln|z_L(t)|) + exp(2 max_{tau in [lo, hi]} ln|z_H(t + tau)|)   (float32)
//   the n_loud largest scores are kept; n_random more times are drawn from the rest
//   (in time order) with numpy's default_rng(seed).integers(0, n_time - n_loud,
//   (n_template, n_random)), each with log weight ln((n_time - n_loud) / n_random);
//   the visited times are returned sorted.
// The score's exp is numpy's float32 exp restated bit for bit (npexp.cuh), so equal trajectories give
// equal scores.  Ties at the n_loud-th score are broken by time (earliest first); numpy's
// argpartition leaves that order unspecified.
#include "common.cuh"
#include "kernels.cuh"
#include "npexp.cuh"
#include "pcg64.cuh"

#define SCORE_TILE 2048

// sliding maximum over the lag window by a sparse table in shared memory, then the score
__global__ void __launch_bounds__(256) k_scores(const float2 *__restrict__ trajH, const float2 *__restrict__ trajL,
                                                 int nt, int lag_lo, int lag_hi, uint32_t *__restrict__ keys)
{
    extern __shared__ float sm_s[];
    const int wn = lag_hi - lag_lo + 1;
    const int L = SCORE_TILE + wn - 1;
    float *a = sm_s, *b = sm_s + L;
    const int m = blockIdx.y;
    const int t0 = blockIdx.x * SCORE_TILE;
    const float2 *H = trajH + (long long)m * nt;
    for (int i = threadIdx.x; i < L; i += blockDim.x) {
        long long t = (long long)t0 + lag_lo + i;
        t %= nt;
        if (t < 0) t += nt;
        a[i] = H[t].x;
    }
    __syncthreads();
    int w = 1;
    while (2 * w <= wn) {
        for (int i = threadIdx.x; i + w < L; i += blockDim.x) b[i] = fmaxf(a[i], a[i + w]);
        __syncthreads();
        float *tmp = a;
        a = b;
        b = tmp;
        w *= 2;
    }
    const float2 *Lr = trajL + (long long)m * nt;
    for (int j = threadIdx.x; j < SCORE_TILE; j += blockDim.x) {
        const int t = t0 + j;
        if (t >= nt) break;
        const float mx = fmaxf(a[j], a[j + wn - w]);
        const float s = __fadd_rn(exm_np_expf(2.0f * Lr[t].x), exm_np_expf(2.0f * mx));
        keys[(long long)m * nt + t] = __float_as_uint(s);
    }
}

// the stream of numpy's bounded integers: 64 draws of 32 bits per thread, rejections listed
// st = {state hi, state lo, inc hi, inc lo} in device memory (staged with the segment's data)
__global__ void k_pcg_draws(const uint64_t *__restrict__ st, long long n_draws, uint32_t range, uint32_t thr,
                            uint32_t *__restrict__ raw, int *__restrict__ rej)
{
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long q0 = g * 64;
    if (q0 >= n_draws) return;
    exm_pcg p;
    p.state = ((exm_u128)st[0] << 64) | st[1];
    p.inc = ((exm_u128)st[2] << 64) | st[3];
    exm_pcg_advance(p, (uint64_t)(g * 32));
    for (int j = 0; j < 32; ++j) {
        exm_pcg_step(p);
        const uint64_t v = exm_pcg_output(p.state);
        for (int h = 0; h < 2; ++h) {
            const long long q = q0 + 2 * j + h;
            if (q >= n_draws) return;
            const uint32_t x = h ? (uint32_t)(v >> 32) : (uint32_t)v;
            const uint64_t mm = (uint64_t)x * range;
            if ((uint32_t)mm < thr) {
                const int c = atomicAdd(rej, 1);
                if (c < EXM_MAX_REJ) rej[1 + c] = (int)q;
                raw[q] = 0xFFFFFFFFu;
            } else {
                raw[q] = (uint32_t)(mm >> 32);
            }
        }
    }
}

// accepted draw o is raw[q] with q = o + (rejections at or before q)
__global__ void k_pcg_compact(const uint32_t *__restrict__ raw, const int *__restrict__ rej, long long n_out,
                              int32_t *__restrict__ picks)
{
    const long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n_out) return;
    const int nrej = min(rej[0], EXM_MAX_REJ);
    long long c = 0;
    for (;;) {
        const long long q = o + c;
        long long c2 = 0;
        for (int i = 0; i < nrej; ++i) c2 += (rej[1 + i] <= q);
        if (c2 == c) {
            picks[o] = (int32_t)raw[q];
            return;
        }
        c = c2;
    }
}

// ------------------------------------------------------------------ top-K, rest draws, merge

__device__ __forceinline__ int block_excl_scan(int v, int *sh, int *total)
{
    // exclusive scan over a block of up to 1024 threads; sh has >= 33 ints
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int s = lane < nw ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) sh[lane] = s;
        if (lane == nw - 1) sh[32] = s;
    }
    __syncthreads();
    const int res = x - v + (warp ? sh[warp - 1] : 0);
    if (total) *total = sh[32];
    __syncthreads();
    return res;
}

__device__ __forceinline__ int lower_bound_i(const int *a, int n, int v)
{
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// one block (1024 threads) per template (internal index i)
__global__ void __launch_bounds__(1024) k_topk(const uint32_t *__restrict__ keys, const int32_t *__restrict__ picks,
                                                const int *__restrict__ order, int nt, int K, int S, int Sp,
                                                int32_t *__restrict__ sel)
{
    extern __shared__ int sm_t[];
    const int nwords = (nt + 31) / 32;
    int *hist = sm_t;                            // 2048
    uint32_t *sbits = (uint32_t *)(hist + 2048); // nwords
    int *zc = (int *)(sbits + nwords);           // nwords + 1
    int *tops = zc + nwords + 1;                 // K
    int *pk = tops + K;                          // Sp
    int *scr = pk + Sp;                          // 40
    const int i = blockIdx.x;
    const uint32_t *key = keys + (long long)i * nt;
    const int tid = threadIdx.x, nth = blockDim.x;

    // radix select of the K-th largest key: digits of 11, 11 and 10 bits from the top
    int kk = K;
    uint32_t prefix = 0, pmask = 0;
    const int shifts[3] = {21, 10, 0}, widths[3] = {11, 11, 10};
    for (int ps = 0; ps < 3; ++ps) {
        const int sh = shifts[ps], nbin = 1 << widths[ps];
        for (int b = tid; b < 2048; b += nth) hist[b] = 0;
        __syncthreads();
        for (int t = tid; t < nt; t += nth) {
            const uint32_t k = key[t];
            if ((k & pmask) == prefix) atomicAdd(&hist[(k >> sh) & (nbin - 1)], 1);
        }
        __syncthreads();
        // suffix sums from the top bin down: each thread owns two adjacent bins
        const int b0 = nbin - 1 - 2 * tid, b1 = b0 - 1;
        const int h0 = (b0 >= 0) ? hist[b0] : 0, h1 = (b1 >= 0) ? hist[b1] : 0;
        int tot;
        const int above = block_excl_scan(h0 + h1, scr, &tot);
        if (b0 >= 0 && above < kk && kk <= above + h0) {
            scr[34] = b0;
            scr[35] = above;
        }
        if (b1 >= 0 && above + h0 < kk && kk <= above + h0 + h1) {
            scr[34] = b1;
            scr[35] = above + h0;
        }
        __syncthreads();
        const int dsel = scr[34];
        kk -= scr[35];
        prefix |= (uint32_t)dsel << sh;
        pmask |= (uint32_t)(nbin - 1) << sh;
        __syncthreads();
    }
    const uint32_t thr = prefix;
    const int need = kk;   // keys equal to thr still to take, earliest first

    // selection mask, built 1024 consecutive times at a time (one bit per time)
    int base_eq = 0;
    for (int c0 = 0; c0 < nwords * 32; c0 += nth) {
        const int t = c0 + tid;
        const uint32_t k = (t < nt) ? key[t] : 0u;
        const int eq = (t < nt) && (k == thr);
        int neq;
        const int r = block_excl_scan(eq, scr, &neq);
        const bool take = (t < nt) && (k > thr || (eq && base_eq + r < need));
        const unsigned bal = __ballot_sync(0xffffffffu, take || t >= nt);  // padding bits count as taken
        if ((tid & 31) == 0 && (t >> 5) < nwords) sbits[t >> 5] = bal;
        base_eq += neq;
    }
    __syncthreads();
    // per-word prefix of selected bits -> the sorted loud times, and the zero (rest) counts
    int carry = 0;
    for (int w0 = 0; w0 < nwords; w0 += nth) {
        const int w = w0 + tid;
        uint32_t bits = (w < nwords) ? sbits[w] : 0u;
        if (w == nwords - 1 && (nt & 31)) bits &= (1u << (nt & 31)) - 1u;   // drop padding
        int tot;
        const int pre = block_excl_scan(__popc(bits), scr, &tot);
        if (w < nwords) {
            const int base = carry + pre;
            zc[w] = w * 32 - base;
            int j = 0;
            while (bits) {
                const int bpos = __ffs(bits) - 1;
                if (base + j < K) tops[base + j] = w * 32 + bpos;
                ++j;
                bits &= bits - 1;
            }
        }
        carry += tot;
    }
    if (tid == 0) zc[nwords] = nt - K;
    __syncthreads();
    // the random draws: rank among the rest (time order) -> time
    const int32_t *prow = picks + (long long)order[i] * S;
    for (int j = tid; j < Sp; j += nth) {
        if (j >= S) {
            pk[j] = 0x7FFFFFFF;
            continue;
        }
        const int p = prow[j];
        int lo = 0, hi = nwords - 1;   // largest w with zc[w] <= p
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (zc[mid] <= p) lo = mid; else hi = mid - 1;
        }
        const int local = p - zc[lo];
        const uint32_t zeros = ~sbits[lo];
        const int bpos = __fns(zeros, 0, local + 1);
        pk[j] = lo * 32 + bpos;
    }
    __syncthreads();
    // bitonic sort of the drawn times (Sp a power of two)
    for (int size = 2; size <= Sp; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int j = tid; j < Sp / 2; j += nth) {
                const int lo2 = 2 * stride * (j / stride) + (j % stride);
                const int hi2 = lo2 + stride;
                const bool up = ((lo2 & size) == 0);
                const int x = pk[lo2], y = pk[hi2];
                if ((x > y) == up) {
                    pk[lo2] = y;
                    pk[hi2] = x;
                }
            }
            __syncthreads();
        }
    }
    // merge: loud times and drawn times are disjoint sets
    int32_t *out = sel + (long long)i * (K + S);
    for (int a = tid; a < K; a += nth) {
        const int t = tops[a];
        const int pos = a + lower_bound_i(pk, S, t);
        if (pos < K + S) out[pos] = t;
    }
    for (int j = tid; j < S; j += nth) {
        const int t = pk[j];
        const int pos = j + lower_bound_i(tops, K, t);
        if (pos < K + S) out[pos] = t | (int)0x80000000;
    }
}

static int next_pow2(int v)
{
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

// the PCG64 state numpy's default_rng(seed) starts from, as {state hi, lo, inc hi, lo}
void exm_pcg_words(uint64_t seed, uint64_t *w)
{
    const exm_pcg g = exm_pcg_from_seed(seed);
    w[0] = (uint64_t)(g.state >> 64);
    w[1] = (uint64_t)g.state;
    w[2] = (uint64_t)(g.inc >> 64);
    w[3] = (uint64_t)g.inc;
}

// the numpy draws of one segment for the whole bank (original template order):
// integers(0, nt - K, size=(nm, S)) from default_rng(seed), the generator state read
// from d_state (4 words on the device).  The raw draws use the key buffer as scratch;
// the selection of each chunk overwrites it afterwards.
void exm_run_pcg(exm_ctx *ctx, exm_slot &sl, const uint64_t *d_state, int K, int S)
{
    const int nt = ctx->nt;
    const uint32_t range = (uint32_t)(nt - K);
    const uint32_t thr = (uint32_t)((1ull << 32) % range);
    const long long n_out = (long long)ctx->nm * S;
    const long long n_draws = ((n_out + EXM_MAX_REJ + 63) / 64) * 64;
    int *rej = (int *)sl.rej.p;
    uint32_t *raw = (uint32_t *)sl.keys.p;
    EXM_CUDA(cudaMemsetAsync(rej, 0, sizeof(int), ctx->stream));
    const long long nthr = n_draws / 64;
    k_pcg_draws<<<(unsigned)((nthr + 127) / 128), 128, 0, ctx->stream>>>(d_state, n_draws, range, thr, raw, rej);
    k_pcg_compact<<<(unsigned)((n_out + 255) / 256), 256, 0, ctx->stream>>>(raw, rej, n_out, (int32_t *)sl.picks.p);
    EXM_CUDA(cudaGetLastError());
    ctx->launches += 2;
}

// scores, top-K, drawn rest times and the sorted merge for the nmc templates of a chunk
void exm_run_topk(exm_ctx *ctx, exm_slot &sl, int nmc, const int *d_order_chunk, int K, int S)
{
    const int nt = ctx->nt;
    const float2 *trajH = (const float2 *)sl.traj.p;
    const float2 *trajL = trajH + (size_t)nmc * nt;
    int lag_lo = (int)ctx->tau[0], lag_hi = (int)ctx->tau[0];
    for (int64_t v : ctx->tau) {
        lag_lo = (int)std::min<int64_t>(lag_lo, v);
        lag_hi = (int)std::max<int64_t>(lag_hi, v);
    }
    const int wn = lag_hi - lag_lo + 1;
    const size_t smem_s = (size_t)2 * (SCORE_TILE + wn - 1) * sizeof(float);
    if (smem_s > 48 * 1024) exm_allow_smem(ctx, (const void *)k_scores, smem_s);
    dim3 gs((nt + SCORE_TILE - 1) / SCORE_TILE, nmc);
    k_scores<<<gs, 256, smem_s, ctx->stream>>>(trajH, trajL, nt, lag_lo, lag_hi, (uint32_t *)sl.keys.p);
    EXM_CUDA(cudaGetLastError());
    const int Sp = next_pow2(std::max(S, 2));
    const int nwords = (nt + 31) / 32;
    const size_t smem_t = sizeof(int) * (2048 + nwords + nwords + 1 + K + Sp + 40);
    if (smem_t > ctx->smem_optin) EXM_THROW(EXM_ERR_ARG, "n_loud + n_random too large for the selection kernel");
    exm_allow_smem(ctx, (const void *)k_topk, smem_t);
    k_topk<<<nmc, 1024, smem_t, ctx->stream>>>((const uint32_t *)sl.keys.p, (const int32_t *)sl.picks.p,
                                               d_order_chunk, nt, K, S, Sp, (int32_t *)sl.sel.p);
    EXM_CUDA(cudaGetLastError());
    ctx->launches += 2;
}

// ------------------------------------------------------------------ the score's exp, for tests

__global__ void k_np_exp32(const float *__restrict__ x, float *__restrict__ y, long long n)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = exm_np_expf(x[i]);
}

void exm_run_np_exp32(exm_ctx *ctx, const float *d_x, float *d_y, long long n)
{
    if (n <= 0) return;
    const long long blocks = std::min<long long>((n + 255) / 256, (long long)ctx->sm_count * 16);
    k_np_exp32<<<(unsigned)blocks, 256, 0, ctx->stream>>>(d_x, d_y, n);
    EXM_CUDA(cudaGetLastError());
}
