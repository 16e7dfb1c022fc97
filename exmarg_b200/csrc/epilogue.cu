// The float64 end of the path:
//  * distance-prior weights per template (exmarg/search/pe.py:260-286, :321-327):
//    'volume' p(y) = 3 ymin^3 y^-4 integrated exactly against a likelihood ratio
//    linear in ln y between the template's points; a tabulated density of ln y
//    ('madau-dickinson') by the trapezoid rule on 401 points per interval;
//  * node values: log-sum-exp over the lags of the per-lag sums, minus ln n_time
//    (gather.py:103-107), then over the nodes with the weights (pe.py:333-336);
//  * ln B: the cell-weighted log-mean over the bank (pe.py:135-142, :338-344).
#include "common.cuh"
#include "kernels.cuh"

#define MAXPTS (EXM_MAX_NODES + 1)

__device__ double interp_density(double t, const double *xp, const double *fp, int n)
{
    // np.interp(t, xp, fp, left=0, right=0)
    if (!(t >= xp[0])) return 0.0;
    if (t > xp[n - 1]) return 0.0;
    if (t == xp[n - 1]) return fp[n - 1];
    int lo = 0, hi = n - 1;   // xp[lo] <= t < xp[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (xp[mid] <= t) lo = mid; else hi = mid;
    }
    const double slope = (fp[lo + 1] - fp[lo]) / (xp[lo + 1] - xp[lo]);
    return slope * (t - xp[lo]) + fp[lo];
}

// y (nn + 1, nm): the template's points (0 where none), internal order; lnW out.  gl (2 x 64: nodes, weights
// on [-1, 1]) non-null: every interval by 64-point Gauss-Legendre in x = ln y, p(x) (b - x) / h and
// p(x) (x - a) / h with p the volume density 3 ymin^3 e^{-3x} or the tabulated one
__global__ void k_distance_weights(const double *__restrict__ y, int nn1, int nm, double ymin, int prior,
                                   const double *__restrict__ lny, const double *__restrict__ plny, int n_dens,
                                   const double *__restrict__ gl, double *__restrict__ lnW)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nm) return;
    int idx[MAXPTS];
    double yy[MAXPTS], w[MAXPTS];
    int np_ = 0;
    for (int k = 0; k < nn1; ++k) {
        const double v = y[(long long)k * nm + i];
        lnW[(long long)k * nm + i] = -INFINITY;
        if (v > 0.0) {
            int pos = np_++;
            while (pos > 0 && yy[pos - 1] > v) {   // insertion by y
                yy[pos] = yy[pos - 1];
                idx[pos] = idx[pos - 1];
                --pos;
            }
            yy[pos] = v;
            idx[pos] = k;
        }
    }
    for (int j = 0; j < np_; ++j) w[j] = 0.0;
    for (int j = 0; j + 1 < np_; ++j) {
        const double a = log(yy[j]), b = log(yy[j + 1]);
        const double h = b - a;
        if (gl) {
            const double c = 3.0 * ymin * ymin * ymin, mid = 0.5 * (a + b), half = 0.5 * h;
            double s0 = 0.0, s1 = 0.0;
            for (int q = 0; q < 64; ++q) {
                const double t = mid + half * gl[q];
                const double f = (prior == EXM_PRIOR_VOLUME) ? c * exp(-3.0 * t) : interp_density(t, lny, plny, n_dens);
                s0 += gl[64 + q] * f * (b - t);
                s1 += gl[64 + q] * f * (t - a);
            }
            w[j] += s0 * half / h;
            w[j + 1] += s1 * half / h;
        } else if (prior == EXM_PRIOR_VOLUME) {
            const double c = 3.0 * ymin * ymin * ymin, kk = 3.0;
            const double ea = exp(-kk * a), eb = exp(-kk * b);
            const double I0 = (ea - eb) / kk;
            const double I1 = (a * ea - b * eb) / kk + (ea - eb) / (kk * kk);
            w[j] += c * (b * I0 - I1) / h;
            w[j + 1] += c * (I1 - a * I0) / h;
        } else {
            const double step = (b - a) / 400.0;
            double s0 = 0.0, s1 = 0.0;
            double tp = a, fp = interp_density(a, lny, plny, n_dens);
            double g0p = fp * (b - tp) / h, g1p = fp * (tp - a) / h;
            for (int q = 1; q <= 400; ++q) {
                const double t = (q == 400) ? b : (double)q * step + a;
                const double f = interp_density(t, lny, plny, n_dens);
                const double g0 = f * (b - t) / h, g1 = f * (t - a) / h;
                const double dx = t - tp;
                s0 += dx * (g0 + g0p) / 2.0;
                s1 += dx * (g1 + g1p) / 2.0;
                tp = t;
                g0p = g0;
                g1p = g1;
            }
            w[j] += s0;
            w[j + 1] += s1;
        }
    }
    for (int j = 0; j < np_; ++j) lnW[(long long)idx[j] * nm + i] = log(w[j]);
}

// ln Lambda per template, and (optionally) the node values lamN (nn + 1, nm)
__global__ void k_node_lse(const double *__restrict__ part, const double *__restrict__ lnW, const int *__restrict__ mlo,
                           const int *__restrict__ mhi, const int *__restrict__ bnode, int nn, int ntau, int nm,
                           int m_base, int nmc, int nt, double *__restrict__ lnl, double *__restrict__ lamN)
{
    const int i = m_base + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m_base + nmc) return;
    const double lnt = log((double)nt);
    double M = -INFINITY, S = 0.0;
    for (int k = 0; k <= nn; ++k) {
        bool valid;
        if (k < nn) valid = (i >= mlo[k] && i < mhi[k]);
        else valid = bnode[i] >= 0;
        double lam = -INFINITY;
        if (valid) {
            const double *pr = part + (long long)k * ntau * nm + i;
            double mx = -INFINITY;
            for (int r = 0; r < ntau; ++r) mx = fmax(mx, pr[(long long)r * nm]);
            double tot = 0.0;
            for (int r = 0; r < ntau; ++r) tot += exp(pr[(long long)r * nm] - mx);
            lam = mx + log(tot) - lnt;
        }
        if (lamN) lamN[(long long)k * nm + i] = lam;
        const double v = lnW[(long long)k * nm + i] + lam;
        if (v > M) {
            S = (M == -INFINITY) ? 1.0 : S * exp(M - v) + 1.0;
            M = v;
        } else if (v > -INFINITY) {
            S += exp(v - M);
        }
    }
    lnl[i] = (M == -INFINITY) ? -INFINITY : M + log(S);
}

// ln B = ln sum_i w_i exp(lnl_i) over the finite terms with w_i > 0 (one block)
__global__ void k_lnb(const double *__restrict__ lnl, const double *__restrict__ cell, int nm, double *__restrict__ out)
{
    __shared__ double sh[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double mx = -INFINITY;
    for (int i = threadIdx.x; i < nm; i += blockDim.x)
        if (isfinite(lnl[i]) && cell[i] > 0.0) mx = fmax(mx, lnl[i]);
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    if (lane == 0) sh[warp] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = -INFINITY;
        for (int q = 0; q < nw; ++q) m = fmax(m, sh[q]);
        sh[0] = m;
    }
    __syncthreads();
    mx = sh[0];
    __syncthreads();
    double s = 0.0;
    if (mx > -INFINITY)
        for (int i = threadIdx.x; i < nm; i += blockDim.x)
            if (isfinite(lnl[i]) && cell[i] > 0.0) s += cell[i] * exp(lnl[i] - mx);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) sh[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < nw; ++q) t += sh[q];
        out[0] = (mx > -INFINITY) ? mx + log(t) : -INFINITY;
    }
}

void exm_run_node_lse(exm_ctx *ctx, exm_slot &sl, int m_base, int nmc)
{
    k_node_lse<<<(nmc + 127) / 128, 128, 0, ctx->stream>>>(
        (const double *)sl.part.p, (const double *)ctx->d_lnW.p, (const int *)ctx->d_mlo.p, (const int *)ctx->d_mhi.p,
        (const int *)ctx->d_bnode.p, ctx->nn, ctx->ntau, ctx->nm, m_base, nmc, ctx->nt, (double *)sl.lnl.p, nullptr);
    EXM_CUDA(cudaGetLastError());
    ctx->launches += 1;
}

void exm_run_node_values(exm_ctx *ctx, exm_slot &sl, double *d_lamN)
{
    k_node_lse<<<(ctx->nm + 127) / 128, 128, 0, ctx->stream>>>(
        (const double *)sl.part.p, (const double *)ctx->d_lnW.p, (const int *)ctx->d_mlo.p, (const int *)ctx->d_mhi.p,
        (const int *)ctx->d_bnode.p, ctx->nn, ctx->ntau, ctx->nm, 0, ctx->nm, ctx->nt, (double *)sl.lnl.p, d_lamN);
    EXM_CUDA(cudaGetLastError());
}

void exm_run_lnb(exm_ctx *ctx, exm_slot &sl)
{
    k_lnb<<<1, 1024, 0, ctx->stream>>>((const double *)sl.lnl.p, (const double *)ctx->d_cell.p, ctx->nm,
                                      (double *)sl.lnb.p);
    EXM_CUDA(cudaGetLastError());
    ctx->launches += 1;
}

void exm_run_distance_weights_y(exm_ctx *ctx, const double *d_y, double ymin, int prior, const double *d_lny,
                                const double *d_p, int n_dens, const double *d_gl)
{
    k_distance_weights<<<(ctx->nm + 127) / 128, 128, 0, ctx->stream>>>(d_y, ctx->nn + 1, ctx->nm, ymin, prior, d_lny,
                                                                       d_p, n_dens, d_gl, (double *)ctx->d_lnW.p);
    EXM_CUDA(cudaGetLastError());
}
