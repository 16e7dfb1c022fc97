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
                const double e = __dadd_rn(__dmul_rn((double)n, be), g[n * kBdTile + j]);
                tot = __dadd_rn(tot, exp(__dsub_rn(e, mx)));
            }
            const float t = (float)__dadd_rn(mx, log(tot));
            T[(size_t)l * per + at] = t;
            bad += !isfinite(t);
        }
    }
    if (bad) atomicAdd(nonfinite, bad);
}

}   // namespace

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
    }
    return 0;
}
