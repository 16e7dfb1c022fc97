// Stage 1 of the offline table build (scripts/build_tables/w_gpu.py:67-182): the GORFs at fixed distance
// at every node s_j, by quadrature over the sky pixels, the polarization angle psi and chi = cos(inclination):
//
//   Wraw_j(tau, (n, a, b)) = sum_pix dep(pix, tau) sum_q Bw_j(q) cos(m dph_q) m1_q^(a+b) m2_q^(2n-a-b),  m = a - b
//   Bw_j(q) = exp(-(s_j |R1|^2 + s_j |R2|^2)) w_q,  m_I = |R_I| / sqrt 2,  dph = arg R1 - arg R2
//   W_j = Wraw_j scale_j(n)
//
// One pixel at a time (its delay deposits on two tau bins, so within a launch every (node, tau, key) is
// written by one block and launches are ordered on the stream: no atomics):
//   k_w_prep: per quadrature point q, the responses R_I in float32 as the reference forms them (products and
//             sums rounded one by one; |R| and arg R rounded to float32 from float64), then in float64 the
//             power ladders m_I^k (k = 0 .. 2 n_max), dph and the damping Bw_j of every node;
//   k_w_gemm: for a phase class m the keys form the triangle pw1 = m + 2x, pw2 = m + 2y, x + y <= n_max - m.
//             A block takes a tile of 8 x-values by 16 y-values (128 keys) and every node (64 rows): a
//             register-tiled float64 GEMM over q in steps of 16, A[j][q] = Bw_j(q) cos(m dph_q) and
//             B[q][(x, y)] = m1_q^pw1 m2_q^pw2 formed in shared memory from the 8 + 16 ladder rows of the tile;
//             the next step's inputs arrive by asynchronous copies (two stages) while a step computes.
//   k_w_scale: W = Wraw * scale, rounded to float32, non-finite entries counted.
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace {

constexpr int kWRows = 64;       // nodes of a tile (n_nodes <= 64)
constexpr int kWX = 8;           // powers of |R1| of a tile
constexpr int kWY = 16;          // powers of |R2| of a tile
constexpr int kWCols = kWX * kWY;
constexpr int kWQ = 16;          // quadrature points per step
constexpr int kWThreads = 128;   // 8 row groups x 16 column groups, 8 x 8 outputs each

__global__ void __launch_bounds__(128) k_w_prep(const float *__restrict__ resp, const float *__restrict__ c2p,
                                                const float *__restrict__ s2p, const float *__restrict__ ap,
                                                const float *__restrict__ cg, const double *__restrict__ wq, int n_psi,
                                                int n_chi, int n_nodes, const double *__restrict__ s, int nl,
                                                double *__restrict__ lad1, double *__restrict__ lad2,
                                                double *__restrict__ dph, double *__restrict__ bw)
{
    const int Q = n_psi * n_chi;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= Q) return;
    const int ip = q / n_chi, ic = q - ip * n_chi;
    float mag[2], ang[2];
    for (int I = 0; I < 2; ++I) {
        const float fp0 = resp[2 * I], fx0 = resp[2 * I + 1];
        const float Fp = __fsub_rn(__fmul_rn(fp0, c2p[ip]), __fmul_rn(fx0, s2p[ip]));
        const float Fx = __fadd_rn(__fmul_rn(fp0, s2p[ip]), __fmul_rn(fx0, c2p[ip]));
        const double re = (double)__fmul_rn(ap[ic], Fp), im = (double)__fmul_rn(cg[ic], Fx);
        mag[I] = (float)sqrt(__dadd_rn(__dmul_rn(re, re), __dmul_rn(im, im)));
        ang[I] = (float)atan2(im, re);
    }
    const double S1 = (double)__fmul_rn(mag[0], mag[0]), S2 = (double)__fmul_rn(mag[1], mag[1]);
    dph[q] = (double)__fsub_rn(ang[0], ang[1]);
    const double m1 = sqrt(S1 / 2.0), m2 = sqrt(S2 / 2.0);
    double a1 = 1.0, a2 = 1.0;
    lad1[q] = 1.0;
    lad2[q] = 1.0;
    for (int k = 1; k < nl; ++k) {
        a1 = __dmul_rn(a1, m1);
        a2 = __dmul_rn(a2, m2);
        lad1[(size_t)k * Q + q] = a1;
        lad2[(size_t)k * Q + q] = a2;
    }
    const double w = wq[ic];
    for (int j = 0; j < n_nodes; ++j)
        bw[(size_t)j * Q + q] = __dmul_rn(exp(-__dadd_rn(__dmul_rn(s[j], S1), __dmul_rn(s[j], S2))), w);
}

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool valid)
{
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(gmem), "r"(valid ? 8 : 0));
}

__global__ void __launch_bounds__(kWThreads, 2) k_w_gemm(const int4 *__restrict__ tiles, int Q, int n_nodes, int n_max,
                                                         const double *__restrict__ lad1, const double *__restrict__ lad2,
                                                         const double *__restrict__ dph, const double *__restrict__ bw,
                                                         int t0, double w0, double w1, int n_tau, long long n_keys,
                                                         double *__restrict__ Wraw)
{
    // two stages of raw inputs filled by asynchronous copies (the next step's while this one computes)
    __shared__ double Ar[2][kWQ][kWRows + 1];       // damping rows, then times cos(m dph) in place
    __shared__ double Ld[2][kWX + kWY][kWQ];        // the tile's |R1| and |R2| ladder rows
    __shared__ double Dp[2][kWQ];
    __shared__ double Bs[kWQ][kWCols + 1];
    __shared__ double cm[kWQ];
    const int4 tl = tiles[blockIdx.x];
    const int m = tl.x, x0 = tl.y, y0 = tl.z;
    const int L = n_max - m + 1;
    const int tid = threadIdx.x, tr = tid >> 4, tc = tid & 15;
    const int nsteps = (Q + kWQ - 1) / kWQ;
    auto issue = [&](int step, int buf) {
        const int q0 = step * kWQ;
        for (int i = tid; i < kWRows * kWQ; i += kWThreads) {
            const int row = i >> 4, qq = i & 15, q = q0 + qq;
            const bool ok = row < n_nodes && q < Q;
            cp_async8(&Ar[buf][qq][row], ok ? bw + (size_t)row * Q + q : bw, ok);
        }
        if (tid < kWQ) {
            const int q = q0 + tid;
            cp_async8(&Dp[buf][tid], q < Q ? dph + q : dph, q < Q);
        } else if (tid < kWQ + (kWX + kWY) * kWQ / 4) {
            for (int i = (tid - kWQ) * 4; i < (tid - kWQ) * 4 + 4; ++i) {
                const int row = i / kWQ, qq = i - row * kWQ, q = q0 + qq;
                if (row < kWX) {
                    const int x = x0 + row;
                    const bool ok = x <= L - 1 && q < Q;
                    cp_async8(&Ld[buf][row][qq], ok ? lad1 + (size_t)(m + 2 * x) * Q + q : lad1, ok);
                } else {
                    const int y = y0 + row - kWX;
                    const bool ok = y <= L - 1 && q < Q;
                    cp_async8(&Ld[buf][row][qq], ok ? lad2 + (size_t)(m + 2 * y) * Q + q : lad2, ok);
                }
            }
        }
        asm volatile("cp.async.commit_group;\n" ::);
    };
    double acc[8][8];
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[r][c] = 0.0;
    issue(0, 0);
    for (int k = 0; k < nsteps; ++k) {
        const int buf = k & 1;
        if (k + 1 < nsteps) issue(k + 1, buf ^ 1);
        else asm volatile("cp.async.commit_group;\n" ::);
        asm volatile("cp.async.wait_group 1;\n" ::);
        __syncthreads();
        if (tid < kWQ) cm[tid] = (k * kWQ + tid < Q) ? cos(__dmul_rn((double)m, Dp[buf][tid])) : 0.0;
        __syncthreads();
        for (int i = tid; i < kWRows * kWQ; i += kWThreads) {
            const int row = i >> 4, qq = i & 15;
            Ar[buf][qq][row] = __dmul_rn(Ar[buf][qq][row], cm[qq]);
        }
        for (int i = tid; i < kWCols * kWQ; i += kWThreads) {
            const int c = i >> 4, qq = i & 15;
            const int x = c >> 4, y = c & 15;   // column c = y + 16 x
            Bs[qq][c] = __dmul_rn(Ld[buf][x][qq], Ld[buf][kWX + y][qq]);
        }
        __syncthreads();
#pragma unroll 4
        for (int qq = 0; qq < kWQ; ++qq) {
            double a[8], b[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) a[r] = Ar[buf][qq][tr + 8 * r];
#pragma unroll
            for (int c = 0; c < 8; ++c) b[c] = Bs[qq][tc + 16 * c];
#pragma unroll
            for (int r = 0; r < 8; ++r)
#pragma unroll
                for (int c = 0; c < 8; ++c) acc[r][c] = fma(a[r], b[c], acc[r][c]);
        }
        __syncthreads();
    }
    asm volatile("cp.async.wait_group 0;\n" ::);
    // thread (tr, tc) holds rows tr + 8 r and columns tc + 16 c: x = x0 + c, y = y0 + tc
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int row = tr + 8 * r;
        if (row >= n_nodes) continue;
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const int x = x0 + c, y = y0 + tc;
            if (x + y > L - 1) continue;
            const long long n = m + x + y, a = m + x, b = x;
            const long long key = n * (n + 1) * (n + 2) / 6 + a * (a + 1) / 2 + b;
            double *dst = Wraw + ((size_t)row * n_tau + t0) * n_keys + key;
            dst[0] = __dadd_rn(dst[0], __dmul_rn(w0, acc[r][c]));
            dst[n_keys] = __dadd_rn(dst[n_keys], __dmul_rn(w1, acc[r][c]));
        }
    }
}

__global__ void k_w_scale(const double *__restrict__ Wraw, const double *__restrict__ scale, int n_tau, long long n_keys,
                          long long n, float *__restrict__ out, unsigned long long *__restrict__ nonfinite)
{
    unsigned long long bad = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long k = i % n_keys, j = i / (n_keys * n_tau);
        const double v = __dmul_rn(Wraw[i], scale[j * n_keys + k]);
        out[i] = (float)v;
        bad += !isfinite(v);
    }
    if (bad) atomicAdd(nonfinite, bad);
}

}   // namespace

extern "C" int exm_w_build(exm_ctx *ctx, int n_nodes, const double *s_nodes, int n_max, int n_psi, int n_chi,
                           const float *c2p, const float *s2p, const float *ap, const float *cg, const double *wq,
                           int n_pix, const float *resp, const int *j0, const double *w, int n_tau, const double *scale,
                           float *W_out, long long *n_nonfinite_out, double *ms_out)
{
    if (!ctx) return EXM_ERR_ARG;
    try {
        EXM_CUDA(cudaSetDevice(ctx->dev));
        if (!(n_nodes >= 1 && n_nodes <= kWRows && n_max >= 0 && n_max <= 255 && n_psi >= 1 && n_chi >= 1 &&
              n_pix >= 1 && n_tau >= 2))
            EXM_THROW(EXM_ERR_ARG, "need 1 <= nodes <= 64, 0 <= n_max <= 255, quadrature and pixels >= 1, n_tau >= 2");
        if (!(s_nodes && c2p && s2p && ap && cg && wq && resp && j0 && w && scale && W_out))
            EXM_THROW(EXM_ERR_ARG, "null argument");
        for (int p = 0; p < n_pix; ++p)
            if (j0[p] < 0 || j0[p] > n_tau - 2) EXM_THROW(EXM_ERR_ARG, "delay bin outside the tau grid");
        const int Q = n_psi * n_chi, nl = 2 * n_max + 1;
        const long long n_keys = (long long)(n_max + 1) * (n_max + 2) * (n_max + 3) / 6;
        std::vector<int4> tiles;
        for (int m = 0; m <= n_max; ++m) {
            const int L = n_max - m + 1;
            for (int x0 = 0; x0 < L; x0 += kWX)
                for (int y0 = 0; x0 + y0 <= L - 1; y0 += kWY) tiles.push_back(make_int4(m, x0, y0, 0));
        }
        const size_t nW = (size_t)n_nodes * n_tau * n_keys;
        dbuf d_s, d_c2p, d_s2p, d_ap, d_cg, d_wq, d_resp, d_scale, d_W, d_out, d_tiles, d_l1, d_l2, d_dph, d_bw, d_bad;
        struct Guard {
            exm_ctx *c;
            std::vector<dbuf *> b;
            ~Guard()
            {
                for (dbuf *x : b)
                    if (x->p) exm_free(c, *x);
            }
        } guard{ctx, {&d_s, &d_c2p, &d_s2p, &d_ap, &d_cg, &d_wq, &d_resp, &d_scale, &d_W, &d_out, &d_tiles, &d_l1,
                      &d_l2, &d_dph, &d_bw, &d_bad}};
        auto up = [&](dbuf &b, const void *src, size_t bytes) {
            exm_alloc(ctx, b, bytes);
            EXM_CUDA(cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
        };
        up(d_s, s_nodes, n_nodes * sizeof(double));
        up(d_c2p, c2p, n_psi * sizeof(float));
        up(d_s2p, s2p, n_psi * sizeof(float));
        up(d_ap, ap, n_chi * sizeof(float));
        up(d_cg, cg, n_chi * sizeof(float));
        up(d_wq, wq, n_chi * sizeof(double));
        up(d_resp, resp, (size_t)n_pix * 4 * sizeof(float));
        up(d_scale, scale, (size_t)n_nodes * n_keys * sizeof(double));
        up(d_tiles, tiles.data(), tiles.size() * sizeof(int4));
        exm_alloc(ctx, d_W, nW * sizeof(double));
        exm_alloc(ctx, d_out, nW * sizeof(float));
        exm_alloc(ctx, d_l1, (size_t)nl * Q * sizeof(double));
        exm_alloc(ctx, d_l2, (size_t)nl * Q * sizeof(double));
        exm_alloc(ctx, d_dph, (size_t)Q * sizeof(double));
        exm_alloc(ctx, d_bw, (size_t)n_nodes * Q * sizeof(double));
        exm_alloc(ctx, d_bad, sizeof(unsigned long long));
        EXM_CUDA(cudaMemsetAsync(d_W.p, 0, nW * sizeof(double), ctx->stream));
        EXM_CUDA(cudaMemsetAsync(d_bad.p, 0, sizeof(unsigned long long), ctx->stream));
        cudaEvent_t e0, e1, e2;
        EXM_CUDA(cudaEventCreate(&e0));
        EXM_CUDA(cudaEventCreate(&e1));
        EXM_CUDA(cudaEventCreate(&e2));
        EXM_CUDA(cudaEventRecord(e0, ctx->stream));
        for (int p = 0; p < n_pix; ++p) {
            k_w_prep<<<(Q + 127) / 128, 128, 0, ctx->stream>>>((const float *)d_resp.p + 4 * (size_t)p,
                                                               (const float *)d_c2p.p, (const float *)d_s2p.p,
                                                               (const float *)d_ap.p, (const float *)d_cg.p,
                                                               (const double *)d_wq.p, n_psi, n_chi, n_nodes,
                                                               (const double *)d_s.p, nl, (double *)d_l1.p,
                                                               (double *)d_l2.p, (double *)d_dph.p, (double *)d_bw.p);
            k_w_gemm<<<(int)tiles.size(), kWThreads, 0, ctx->stream>>>(
                (const int4 *)d_tiles.p, Q, n_nodes, n_max, (const double *)d_l1.p, (const double *)d_l2.p,
                (const double *)d_dph.p, (const double *)d_bw.p, j0[p], w[2 * p], w[2 * p + 1], n_tau, n_keys,
                (double *)d_W.p);
        }
        EXM_CUDA(cudaGetLastError());
        EXM_CUDA(cudaEventRecord(e1, ctx->stream));
        k_w_scale<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>((const double *)d_W.p, (const double *)d_scale.p, n_tau,
                                                              n_keys, (long long)nW, (float *)d_out.p,
                                                              (unsigned long long *)d_bad.p);
        EXM_CUDA(cudaGetLastError());
        unsigned long long bad = 0;
        EXM_CUDA(cudaMemcpyAsync(W_out, d_out.p, nW * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
        EXM_CUDA(cudaMemcpyAsync(&bad, d_bad.p, sizeof(bad), cudaMemcpyDeviceToHost, ctx->stream));
        EXM_CUDA(cudaEventRecord(e2, ctx->stream));
        EXM_CUDA(cudaStreamSynchronize(ctx->stream));
        float k_ms = 0.f, all_ms = 0.f;
        cudaEventElapsedTime(&k_ms, e0, e1);
        cudaEventElapsedTime(&all_ms, e0, e2);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaEventDestroy(e2);
        if (n_nonfinite_out) *n_nonfinite_out = (long long)bad;
        if (ms_out) {
            ms_out[0] = k_ms;
            ms_out[1] = all_ms;
        }
        ctx->launches += 2 * n_pix + 1;
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
