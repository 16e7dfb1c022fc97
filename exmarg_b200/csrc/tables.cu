// The offline table build, stage 3 (scripts/build_tables/build_bd.py:53-77): the log-sum over the
// orders n of the series that gives a node's table T[tau, phi+, beta, Delta].
//
// Every order is homogeneous, lnK_n(q1, q2) = 2n ln q2 + g_n(ln q1 - ln q2), so the sum
//     T(beta, Delta) = log sum_n exp(n beta + g_n(Delta))
// needs g_n only on the last column (q2 = q_last: Delta <= 0) and the last row (q1 = q_last:
// Delta >= 0) of each (q1, q2) block of stage 2:
//     g_n(Delta_i)          = col[n, tau, q1 = i, phi] - 2n ln q_last          i = 0 .. nq-1
//     g_n(Delta_{nq-1+j})   = row[n, tau, q2 = nq-1-j, phi] - 2n ln q_{nq-1-j}  j = 1 .. nq-1
// One block per (tau, phi, tile of Delta): the tile's g_n for every order in shared memory, then each
// thread takes (beta, Delta) outputs: the maximum over the orders up to each truncation order, then
// the sum of exp(E - max) in order of n, in float64 with the products and sums rounded one by one
// as numpy evaluates them (no fused multiply-add), rounded to float32 at the end.
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace {

constexpr int kBdTile = 32;   // Delta columns per block

__global__ void __launch_bounds__(256) k_bd_lse(const float *__restrict__ col, const float *__restrict__ row,
                                                const double *__restrict__ lnq, int nord, int ntau, int nq, int nphif,
                                                const double *__restrict__ beta, int nb, const int *__restrict__ ladder,
                                                int nl, float *__restrict__ T, unsigned long long *__restrict__ nonfinite)
{
    const int nd = 2 * nq - 1;
    const int ntile = (nd + kBdTile - 1) / kBdTile;
    int blk = blockIdx.x;
    const int tile = blk % ntile;
    blk /= ntile;
    const int pi = blk % nphif;
    const int ti = blk / nphif;
    extern __shared__ double g[];   // [nord][kBdTile]
    const int d0 = tile * kBdTile;
    const int dn = min(kBdTile, nd - d0);
    const double lq_last = lnq[nq - 1];
    for (int i = threadIdx.x; i < nord * kBdTile; i += blockDim.x) {
        const int n = i / kBdTile, j = i - n * kBdTile, d = d0 + j;
        const double two_n = 2.0 * (double)n;
        double v = 0.0;
        if (j < dn) {
            if (d < nq) {
                const double c = (double)col[(((size_t)n * ntau + ti) * nq + d) * nphif + pi];
                v = __dsub_rn(c, __dmul_rn(two_n, lq_last));
            } else {
                const int q2 = 2 * nq - 2 - d;
                const double r = (double)row[(((size_t)n * ntau + ti) * nq + q2) * nphif + pi];
                v = __dsub_rn(r, __dmul_rn(two_n, lnq[q2]));
            }
        }
        g[i] = v;
    }
    __syncthreads();
    const size_t per = (size_t)ntau * nphif * nb * nd;
    unsigned long long bad = 0;
    for (int o = threadIdx.x; o < nb * dn; o += blockDim.x) {
        const int b = o / dn, j = o - b * dn;
        const double be = beta[b];
        const size_t at = (((size_t)ti * nphif + pi) * nb + b) * nd + d0 + j;
        for (int l = 0; l < nl; ++l) {
            const int nm = ladder[l];
            double mx = -INFINITY;
            for (int n = 0; n <= nm; ++n) mx = fmax(mx, __dadd_rn(__dmul_rn((double)n, be), g[n * kBdTile + j]));
            double tot = 0.0;
            for (int n = 0; n <= nm; ++n) {
                const double e = __dsub_rn(__dadd_rn(__dmul_rn((double)n, be), g[n * kBdTile + j]), mx);
                if (!(e <= -746.0)) tot = __dadd_rn(tot, exp(e));   // below, exp is exactly 0 (a NaN still adds)
            }
            const float t = (float)__dadd_rn(mx, log(tot));
            T[(size_t)l * per + at] = t;
            bad += !isfinite(t);
        }
    }
    if (bad) atomicAdd(nonfinite, bad);
}

// Stage 2 on the boundary only (scripts/build_tables/build_k.py:59-82 restricted to q2 = q_last, the
// column, and q1 = q_last, the row, which is all stage 3 reads): for order n and phase class m = a - b,
//   C_m(tau, qb) = sum_{a - b = m} c_ab W_ab(tau) exp((a + b) lq1 + (2n - a - b) lq2 - 2n lq_last)
// with c_ab = C(n, a) C(n, b) (2 if m > 0), qb running over the column (lq1 = lnq[qb], lq2 = lq_last) then
// the row (lq1 = lq_last, lq2 = lnq[qb - nq], qb - nq < nq - 1).  One block per (n, m, 8 lags); the
// exponentials of 16 rows at a time in shared memory; each thread holds at most 8 of the block's
// 8 x (2 nq - 1) outputs.
constexpr int kKTau = 8;
constexpr int kKRows = 16;

__global__ void __launch_bounds__(256) k_k_class(const double *__restrict__ Wd, const double *__restrict__ coeff,
                                                 const int2 *__restrict__ cls, int n_tau, int nq,
                                                 const double *__restrict__ lnq, double *__restrict__ C)
{
    const int nqb = 2 * nq - 1;
    const int ntc = (n_tau + kKTau - 1) / kKTau;
    const int c = blockIdx.x / ntc, t0 = (blockIdx.x - c * ntc) * kKTau;
    const int2 nm = cls[c];   // (n, m)
    const int n = nm.x, m = nm.y, nrows = n - m + 1;
    const long long key0 = (long long)n * (n + 1) * (n + 2) / 6;
    __shared__ double P[kKRows][2 * 128];   // nq <= 128
    __shared__ double Wm[kKRows][kKTau];
    const double lql = lnq[nq - 1];
    const double g = __dmul_rn(2.0 * (double)n, lql);
    const int nout = kKTau * nqb;   // <= 8 * 256
    double acc[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) acc[k] = 0.0;
    for (int r0 = 0; r0 < nrows; r0 += kKRows) {
        const int rn = min(kKRows, nrows - r0);
        __syncthreads();
        for (int i = threadIdx.x; i < rn * nqb; i += blockDim.x) {
            const int r = i / nqb, qb = i - r * nqb;
            const int a = m + r0 + r, b = a - m;
            const double lq1 = qb < nq ? lnq[qb] : lql, lq2 = qb < nq ? lql : lnq[qb - nq];
            const double e = __dsub_rn(__dadd_rn(__dmul_rn((double)(a + b), lq1), __dmul_rn((double)(2 * n - a - b), lq2)), g);
            P[r][qb] = exp(e);
        }
        for (int i = threadIdx.x; i < rn * kKTau; i += blockDim.x) {
            const int r = i / kKTau, tt = i - r * kKTau, t = t0 + tt;
            const int a = m + r0 + r, b = a - m;
            const long long key = key0 + (long long)a * (a + 1) / 2 + b;
            Wm[r][tt] = t < n_tau ? __dmul_rn(coeff[key], Wd[key * n_tau + t]) : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int o = threadIdx.x + k * 256;
            if (o < nout) {
                const int tt = o / nqb, qb = o - tt * nqb;
                double v = acc[k];
                for (int r = 0; r < rn; ++r) v = fma(Wm[r][tt], P[r][qb], v);
                acc[k] = v;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int o = threadIdx.x + k * 256;
        if (o < nout) {
            const int tt = o / nqb, qb = o - tt * nqb, t = t0 + tt;
            if (t < n_tau) C[((long long)c * n_tau + t) * nqb + qb] = acc[k];
        }
    }
}

// K_n(tau, qb, phi) = sum_m cos(m phi) C_m(tau, qb); lnK = float32(log(max(K_n, 1e-300)) + (2n lq_last - o_n))
// into the column col[n][tau][q1][phi] and the row row[n][tau][q2][phi] (the corner q1 = q2 = q_last in both)
__global__ void __launch_bounds__(256) k_k_phase(const double *__restrict__ C, const int *__restrict__ cls0, int n_tau,
                                                 int nq, int nphif, const double *__restrict__ cosm, int ncos,
                                                 const double *__restrict__ gmo, float *__restrict__ col,
                                                 float *__restrict__ row)
{
    const int nqb = 2 * nq - 1;
    const int n = blockIdx.x / n_tau, t = blockIdx.x - n * n_tau;
    const int c0 = cls0[n];   // class index of (n, 0); the classes of n are c0 .. c0 + n
    for (int o = threadIdx.x; o < nqb * nphif; o += blockDim.x) {
        const int qb = o / nphif, p = o - qb * nphif;
        double K = 0.0;
        for (int m = 0; m <= n; ++m)
            K = fma(cosm[(long long)m * ncos + p], C[((long long)(c0 + m) * n_tau + t) * nqb + qb], K);
        const float v = (float)__dadd_rn(log(fmax(K, 1e-300)), gmo[n]);
        const long long base = ((long long)n * n_tau + t) * nq;
        if (qb < nq) {
            col[(base + qb) * nphif + p] = v;
            if (qb == nq - 1) row[(base + qb) * nphif + p] = v;
        } else {
            row[(base + qb - nq) * nphif + p] = v;
        }
    }
}

}   // namespace

extern "C" int exm_k_edges(exm_ctx *ctx, int n_max, int n_tau, const double *Wd, const double *coeff, int nq,
                           const double *lnq, const double *gmo, int nphif, const double *cosm, float *col_out,
                           float *row_out, double *ms_out)
{
    if (!ctx) return EXM_ERR_ARG;
    try {
        EXM_CUDA(cudaSetDevice(ctx->dev));
        if (!(n_max >= 0 && n_max <= 255 && n_tau >= 1 && nq >= 2 && nq <= 128 && nphif >= 1))
            EXM_THROW(EXM_ERR_ARG, "need 0 <= n_max <= 255, lags >= 1, 2 <= nq <= 128, phases >= 1");
        if (!(Wd && coeff && lnq && gmo && cosm && col_out && row_out)) EXM_THROW(EXM_ERR_ARG, "null argument");
        const long long n_keys = (long long)(n_max + 1) * (n_max + 2) * (n_max + 3) / 6;
        std::vector<int2> cls;
        std::vector<int> cls0(n_max + 1);
        for (int n = 0; n <= n_max; ++n) {
            cls0[n] = (int)cls.size();
            for (int m = 0; m <= n; ++m) cls.push_back(make_int2(n, m));
        }
        const int nqb = 2 * nq - 1;
        const size_t nC = cls.size() * (size_t)n_tau * nqb, nE = (size_t)(n_max + 1) * n_tau * nq * nphif;
        dbuf dW, dco, dlnq, dgmo, dcos, dcls, dcls0, dC, dcol, drow;
        struct Guard {
            exm_ctx *c;
            std::vector<dbuf *> b;
            ~Guard()
            {
                for (dbuf *x : b)
                    if (x->p) exm_free(c, *x);
            }
        } guard{ctx, {&dW, &dco, &dlnq, &dgmo, &dcos, &dcls, &dcls0, &dC, &dcol, &drow}};
        auto up = [&](dbuf &b, const void *src, size_t bytes) {
            exm_alloc(ctx, b, bytes);
            EXM_CUDA(cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
        };
        cudaEvent_t e0, e1;
        EXM_CUDA(cudaEventCreate(&e0));
        EXM_CUDA(cudaEventCreate(&e1));
        up(dW, Wd, (size_t)n_keys * n_tau * sizeof(double));
        up(dco, coeff, (size_t)n_keys * sizeof(double));
        up(dlnq, lnq, nq * sizeof(double));
        up(dgmo, gmo, (n_max + 1) * sizeof(double));
        up(dcos, cosm, (size_t)(n_max + 1) * nphif * sizeof(double));
        up(dcls, cls.data(), cls.size() * sizeof(int2));
        up(dcls0, cls0.data(), cls0.size() * sizeof(int));
        exm_alloc(ctx, dC, nC * sizeof(double));
        exm_alloc(ctx, dcol, nE * sizeof(float));
        exm_alloc(ctx, drow, nE * sizeof(float));
        EXM_CUDA(cudaEventRecord(e0, ctx->stream));
        const long long nblk = (long long)cls.size() * ((n_tau + kKTau - 1) / kKTau);
        k_k_class<<<(int)nblk, 256, 0, ctx->stream>>>((const double *)dW.p, (const double *)dco.p, (const int2 *)dcls.p,
                                                      n_tau, nq, (const double *)dlnq.p, (double *)dC.p);
        k_k_phase<<<(n_max + 1) * n_tau, 256, 0, ctx->stream>>>((const double *)dC.p, (const int *)dcls0.p, n_tau, nq,
                                                                nphif, (const double *)dcos.p, nphif,
                                                                (const double *)dgmo.p, (float *)dcol.p, (float *)drow.p);
        EXM_CUDA(cudaGetLastError());
        EXM_CUDA(cudaEventRecord(e1, ctx->stream));
        EXM_CUDA(cudaMemcpyAsync(col_out, dcol.p, nE * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
        EXM_CUDA(cudaMemcpyAsync(row_out, drow.p, nE * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
        EXM_CUDA(cudaStreamSynchronize(ctx->stream));
        float k_ms = 0.f;
        cudaEventElapsedTime(&k_ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (ms_out) ms_out[0] = k_ms;
        ctx->launches += 2;
    } catch (const exm_error &e) {
        ctx->err = e.msg;
        return e.code;
    } catch (const std::bad_alloc &) {
        ctx->err = "host memory exhausted";
        return EXM_ERR_OOM;
    } catch (const std::exception &e) {
        ctx->err = e.what();
        return EXM_ERR_CUDA;
    }
    return 0;
}

extern "C" int exm_bd_build(exm_ctx *ctx, int nord, int ntau, int nq, int nphif, const float *col, const float *row,
                            const double *lnq, int nb, const double *beta, int n_ladder, const int *ladder,
                            float *T_out, long long *n_nonfinite, double *ms_out)
{
    if (!ctx) return EXM_ERR_ARG;
    try {
        EXM_CUDA(cudaSetDevice(ctx->dev));
        if (!(nord >= 1 && nord <= 256 && ntau >= 1 && nq >= 2 && nq <= 4096 && nphif >= 1 && nb >= 1))
            EXM_THROW(EXM_ERR_ARG, "need 1 <= orders <= 256, lags >= 1, 2 <= nq <= 4096, phases >= 1, nb >= 1");
        if (!(col && row && lnq && beta && ladder && T_out && n_ladder >= 1)) EXM_THROW(EXM_ERR_ARG, "null argument");
        for (int l = 0; l < n_ladder; ++l)
            if (ladder[l] < 0 || ladder[l] >= nord) EXM_THROW(EXM_ERR_ARG, "truncation orders must lie in 0 .. orders-1");
        const int nd = 2 * nq - 1;
        const size_t nin = (size_t)nord * ntau * nq * nphif, per = (size_t)ntau * nphif * nb * nd;
        dbuf dcol, drow, dlnq, dbeta, dlad, dT, dbad;
        struct Guard {
            exm_ctx *c;
            dbuf *b[7];
            ~Guard()
            {
                for (dbuf *x : b)
                    if (x->p) exm_free(c, *x);
            }
        } guard{ctx, {&dcol, &drow, &dlnq, &dbeta, &dlad, &dT, &dbad}};
        exm_alloc(ctx, dcol, nin * sizeof(float));
        exm_alloc(ctx, drow, nin * sizeof(float));
        exm_alloc(ctx, dlnq, nq * sizeof(double));
        exm_alloc(ctx, dbeta, nb * sizeof(double));
        exm_alloc(ctx, dlad, n_ladder * sizeof(int));
        exm_alloc(ctx, dT, (size_t)n_ladder * per * sizeof(float));
        exm_alloc(ctx, dbad, sizeof(unsigned long long));
        cudaEvent_t e0, e1, e2, e3;
        EXM_CUDA(cudaEventCreate(&e0));
        EXM_CUDA(cudaEventCreate(&e1));
        EXM_CUDA(cudaEventCreate(&e2));
        EXM_CUDA(cudaEventCreate(&e3));
        EXM_CUDA(cudaEventRecord(e0, ctx->stream));
        EXM_CUDA(cudaMemcpyAsync(dcol.p, col, nin * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
        EXM_CUDA(cudaMemcpyAsync(drow.p, row, nin * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
        EXM_CUDA(cudaMemcpyAsync(dlnq.p, lnq, nq * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        EXM_CUDA(cudaMemcpyAsync(dbeta.p, beta, nb * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        EXM_CUDA(cudaMemcpyAsync(dlad.p, ladder, n_ladder * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
        EXM_CUDA(cudaMemsetAsync(dbad.p, 0, sizeof(unsigned long long), ctx->stream));
        const size_t smem = (size_t)nord * kBdTile * sizeof(double);
        exm_allow_smem(ctx, (const void *)k_bd_lse, smem);
        const long long nblk = (long long)ntau * nphif * ((nd + kBdTile - 1) / kBdTile);
        if (nblk > 0x7fffffffLL) EXM_THROW(EXM_ERR_ARG, "table too large");
        EXM_CUDA(cudaEventRecord(e1, ctx->stream));
        k_bd_lse<<<(int)nblk, 256, smem, ctx->stream>>>((const float *)dcol.p, (const float *)drow.p,
                                                        (const double *)dlnq.p, nord, ntau, nq, nphif,
                                                        (const double *)dbeta.p, nb, (const int *)dlad.p, n_ladder,
                                                        (float *)dT.p, (unsigned long long *)dbad.p);
        EXM_CUDA(cudaGetLastError());
        EXM_CUDA(cudaEventRecord(e2, ctx->stream));
        unsigned long long bad = 0;
        EXM_CUDA(cudaMemcpyAsync(T_out, dT.p, (size_t)n_ladder * per * sizeof(float), cudaMemcpyDeviceToHost,
                                 ctx->stream));
        EXM_CUDA(cudaMemcpyAsync(&bad, dbad.p, sizeof(bad), cudaMemcpyDeviceToHost, ctx->stream));
        EXM_CUDA(cudaEventRecord(e3, ctx->stream));
        EXM_CUDA(cudaStreamSynchronize(ctx->stream));
        float k_ms = 0.f, all_ms = 0.f;
        cudaEventElapsedTime(&k_ms, e1, e2);
        cudaEventElapsedTime(&all_ms, e0, e3);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaEventDestroy(e2);
        cudaEventDestroy(e3);
        if (n_nonfinite) *n_nonfinite = (long long)bad;
        if (ms_out) {
            ms_out[0] = k_ms;
            ms_out[1] = all_ms;
        }
        ctx->launches += 1;
    } catch (const exm_error &e) {
        ctx->err = e.msg;
        return e.code;
    } catch (const std::bad_alloc &) {
        ctx->err = "host memory exhausted";
        return EXM_ERR_OOM;
    } catch (const std::exception &e) {
        ctx->err = e.what();
        return EXM_ERR_CUDA;
    }
    return 0;
}
