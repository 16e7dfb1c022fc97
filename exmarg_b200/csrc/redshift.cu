// The source frame of pe_redshift (exmarg/search/pe.py:87-132, _to_source_frame, and the ln B of
// :249-255): a segment's node values ln Lambda(node, template) become ln Lambda on an (m1, z) grid,
// linear in y = D0 / D_L per template between its finite node values, then linear in the
// detector-frame total mass M_det = 2 m1 (1 + z) per z between the templates finite there; ln B is
// the prior-weighted mean over the grid.  Float64 throughout, each interpolation with the
// reference's operations in its order (no fused multiply-add), so the device surface equals the
// reference's for the same node values.
//
// k_rs_surf: one block per template: its finite (y, ln Lambda) points sorted by y in shared memory,
//            then every z of the grid.
// k_rs_out:  one block per z: the templates finite at that z (a block-wide scan), then every m1.
// k_rs_lnb:  one block: the log of the weighted mean, max then sum.
#include <cmath>

#include "common.cuh"
#include "kernels.cuh"

struct exm_redshift {
    int nn1 = 0, nm = 0, nz = 0, nm1 = 0;
    dbuf yN, M, yq, z, m1, w;   // [nn1][nm], [nm], [nz], [nz], [nm1], [nm1][nz]
    dbuf lamN, surf, out, red;  // [nn1][nm], [nz][nm], [nm1][nz], 2 doubles
};

#define EXM_RS_MAX_POINTS (EXM_MAX_NODES + 1)
#define EXM_RS_MAX_TEMPLATES 8192

__global__ void __launch_bounds__(128) k_rs_surf(const double *__restrict__ lamN, const double *__restrict__ yN,
                                                 int nn1, int nm, const double *__restrict__ yq, int nz,
                                                 double *__restrict__ surf)
{
    __shared__ double ys[EXM_RS_MAX_POINTS], ls[EXM_RS_MAX_POINTS];
    __shared__ int n_sh;
    const int m = blockIdx.x;
    if (threadIdx.x == 0) {
        int n = 0;
        for (int k = 0; k < nn1; ++k) {   // the finite points with y > 0, insertion-sorted by y
            const double L = lamN[(long long)k * nm + m], Y = yN[(long long)k * nm + m];
            if (!(isfinite(L) && Y > 0.0)) continue;
            int i = n++;
            while (i > 0 && ys[i - 1] > Y) {
                ys[i] = ys[i - 1];
                ls[i] = ls[i - 1];
                --i;
            }
            ys[i] = Y;
            ls[i] = L;
        }
        n_sh = n;
    }
    __syncthreads();
    const int n = n_sh;
    for (int iz = threadIdx.x; iz < nz; iz += blockDim.x) {
        double v = -INFINITY;
        if (n >= 2) {
            const double q = yq[iz];
            int cnt = 0;
            for (int i = 0; i < n; ++i) cnt += ys[i] <= q;
            const int lo = min(max(cnt - 1, 0), n - 2), hi = lo + 1;
            const double y0 = ys[lo], y1 = ys[hi], v0 = ls[lo], v1 = ls[hi];
            const double t = y1 > y0 ? __ddiv_rn(__dsub_rn(q, y0), __dsub_rn(y1, y0)) : 1.0;
            if (q >= ys[0] && q <= ys[n - 1]) v = __dadd_rn(v0, __dmul_rn(t, __dsub_rn(v1, v0)));
        }
        surf[(long long)iz * nm + m] = v;
    }
}

__global__ void __launch_bounds__(256) k_rs_out(const double *__restrict__ surf, int nm, const double *__restrict__ M,
                                                const double *__restrict__ z, int nz, const double *__restrict__ m1,
                                                int nm1, double *__restrict__ out)
{
    extern __shared__ int rs_sm[];
    int *rank = rs_sm;        // [nm]: templates finite at this z up to and including each one
    int *G = rs_sm + nm;      // [nm]: index of the r-th finite template
    __shared__ int wsum[8], carry_sh;
    const int iz = blockIdx.x;
    const double *s = surf + (long long)iz * nm;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry_sh = 0;
    __syncthreads();
    for (int b = 0; b < nm; b += blockDim.x) {   // block-wide inclusive scan of the finite flags
        const int m = b + threadIdx.x;
        const int g = (m < nm && isfinite(s[m])) ? 1 : 0;
        int x = g;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[warp] = x;
        __syncthreads();
        int pre = carry_sh;
        for (int w = 0; w < warp; ++w) pre += wsum[w];
        if (m < nm) {
            rank[m] = pre + x;
            if (g) G[pre + x - 1] = m;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += wsum[w];
            carry_sh += t;
        }
        __syncthreads();
    }
    const int ngood = carry_sh;
    if (ngood == 0 && threadIdx.x == 0) G[0] = 0;
    __syncthreads();
    const double zp1 = __dadd_rn(1.0, z[iz]);
    const int glast = G[max(ngood - 1, 0)];
    const double first = M[G[0]], last = M[glast];
    for (int i1 = threadIdx.x; i1 < nm1; i1 += blockDim.x) {
        const double Md = __dmul_rn(__dmul_rn(2.0, m1[i1]), zp1);
        int p = 0, hi_s = nm;   // p = number of masses below Md (searchsorted, left)
        while (p < hi_s) {
            const int mid = (p + hi_s) >> 1;
            if (M[mid] < Md) p = mid + 1; else hi_s = mid;
        }
        const int below = p > 0 ? rank[p - 1] : 0;
        const int hi = G[min(below, max(ngood - 1, 0))];
        const int lo = below >= 1 ? G[max(below - 1, 0)] : hi;
        const double m0 = M[lo], mh = M[hi], w0 = s[lo], w1 = s[hi];
        const double t = mh > m0 ? __ddiv_rn(__dsub_rn(Md, m0), __dsub_rn(mh, m0)) : 0.0;
        const bool inb = ngood >= 2 && Md >= first && Md <= last;
        out[(long long)i1 * nz + iz] = inb ? __dadd_rn(w0, __dmul_rn(t, __dsub_rn(w1, w0))) : -INFINITY;
    }
}

// ln sum_i w_i exp(L_i) over the finite L with w > 0 (exmarg/search/pe.py:135-142); red[0] = ln B
__global__ void __launch_bounds__(1024) k_rs_lnb(const double *__restrict__ L, const double *__restrict__ w,
                                                 long long n, double *__restrict__ red)
{
    __shared__ double sh[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double mx = -INFINITY;
    for (long long i = threadIdx.x; i < n; i += blockDim.x)
        if (isfinite(L[i]) && w[i] > 0.0) mx = fmax(mx, L[i]);
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) sh[warp] = mx;
    __syncthreads();
    if (warp == 0) {
        double v = lane < (int)(blockDim.x >> 5) ? sh[lane] : -INFINITY;
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0) sh[0] = v;
    }
    __syncthreads();
    mx = sh[0];
    __syncthreads();
    double acc = 0.0;
    if (isfinite(mx))
        for (long long i = threadIdx.x; i < n; i += blockDim.x)
            if (isfinite(L[i]) && w[i] > 0.0) acc += w[i] * exp(L[i] - mx);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) sh[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += sh[q];
        red[0] = isfinite(mx) ? mx + log(t) : -INFINITY;
    }
}

void exm_redshift_release(exm_ctx *ctx)
{
    exm_redshift *r = ctx->rs;
    if (!r) return;
    dbuf *all[] = {&r->yN, &r->M, &r->yq, &r->z, &r->m1, &r->w, &r->lamN, &r->surf, &r->out, &r->red};
    for (dbuf *b : all) exm_free(ctx, *b);
    delete r;
    ctx->rs = nullptr;
}

extern "C" int exm_redshift_grid(exm_ctx *ctx, int nn1, int nm, const double *yN, const double *Mdet, int nz,
                                 const double *yq, const double *z, int nm1, const double *m1, const double *w)
{
    if (!ctx) return EXM_ERR_ARG;
    try {
        EXM_CUDA(cudaSetDevice(ctx->dev));
        if (nn1 < 2 || nn1 > EXM_RS_MAX_POINTS) EXM_THROW(EXM_ERR_ARG, "nn1 (nodes + boundary row) must be 2..65");
        if (nm < 1 || nm > EXM_RS_MAX_TEMPLATES) EXM_THROW(EXM_ERR_ARG, "the bank must have 1..8192 templates");
        if (nz < 1 || nm1 < 1) EXM_THROW(EXM_ERR_ARG, "empty (m1, z) grid");
        if (!yN || !Mdet || !yq || !z || !m1 || !w) EXM_THROW(EXM_ERR_ARG, "null grid array");
        for (int i = 1; i < nm; ++i)
            if (!(Mdet[i] > Mdet[i - 1])) EXM_THROW(EXM_ERR_ARG, "detector-frame masses must ascend");
        exm_redshift_release(ctx);
        exm_redshift *r = new exm_redshift();
        ctx->rs = r;
        r->nn1 = nn1;
        r->nm = nm;
        r->nz = nz;
        r->nm1 = nm1;
        auto up = [&](dbuf &b, const double *src, size_t n) {
            exm_alloc(ctx, b, n * sizeof(double));
            EXM_CUDA(cudaMemcpyAsync(b.p, src, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        };
        up(r->yN, yN, (size_t)nn1 * nm);
        up(r->M, Mdet, nm);
        up(r->yq, yq, nz);
        up(r->z, z, nz);
        up(r->m1, m1, nm1);
        up(r->w, w, (size_t)nm1 * nz);
        exm_alloc(ctx, r->lamN, sizeof(double) * nn1 * nm);
        exm_alloc(ctx, r->surf, sizeof(double) * (size_t)nz * nm);
        exm_alloc(ctx, r->out, sizeof(double) * (size_t)nm1 * nz);
        exm_alloc(ctx, r->red, 2 * sizeof(double));
        exm_allow_smem(ctx, (const void *)k_rs_out, 2 * sizeof(int) * (size_t)nm);
        EXM_CUDA(cudaStreamSynchronize(ctx->stream));
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
    return EXM_OK;
}

extern "C" int exm_source_frame(exm_ctx *ctx, const double *lamN, double *ln_lambda_out, double *ln_b_out)
{
    if (!ctx) return EXM_ERR_ARG;
    try {
        EXM_CUDA(cudaSetDevice(ctx->dev));
        exm_redshift *r = ctx->rs;
        if (!r) EXM_THROW(EXM_ERR_STATE, "exm_redshift_grid first");
        if (!lamN) EXM_THROW(EXM_ERR_ARG, "null node values");
        EXM_CUDA(cudaMemcpyAsync(r->lamN.p, lamN, sizeof(double) * r->nn1 * r->nm, cudaMemcpyHostToDevice,
                                 ctx->stream));
        k_rs_surf<<<r->nm, 128, 0, ctx->stream>>>((const double *)r->lamN.p, (const double *)r->yN.p, r->nn1, r->nm,
                                                  (const double *)r->yq.p, r->nz, (double *)r->surf.p);
        k_rs_out<<<r->nz, 256, 2 * sizeof(int) * (size_t)r->nm, ctx->stream>>>(
            (const double *)r->surf.p, r->nm, (const double *)r->M.p, (const double *)r->z.p, r->nz,
            (const double *)r->m1.p, r->nm1, (double *)r->out.p);
        k_rs_lnb<<<1, 1024, 0, ctx->stream>>>((const double *)r->out.p, (const double *)r->w.p,
                                              (long long)r->nm1 * r->nz, (double *)r->red.p);
        EXM_CUDA(cudaGetLastError());
        ctx->launches += 3;
        if (ln_lambda_out)
            EXM_CUDA(cudaMemcpyAsync(ln_lambda_out, r->out.p, sizeof(double) * (size_t)r->nm1 * r->nz,
                                     cudaMemcpyDeviceToHost, ctx->stream));
        double lnb = 0.0;
        EXM_CUDA(cudaMemcpyAsync(&lnb, r->red.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        EXM_CUDA(cudaStreamSynchronize(ctx->stream));
        if (ln_b_out) *ln_b_out = lnb;
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
    return EXM_OK;
}
