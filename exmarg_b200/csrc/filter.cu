// Matched filter of one segment against the whole bank (exmarg/search/bank.py:56-78):
//   w_I = complex64(conj(d_I) / sig2_I)          (float64 division, rounded once)
//   pad[m, lo:lo+nf] = W[m] * w_I                 (complex64 product, no FMA contraction)
//   z = FFT_forward(pad)                          (cuFFT C2C, length n_time, batched)
//   (ln|z|, arg z) = (0.5 ln max(re^2 + im^2, 1e-38), atan2(im, re))
// The pre-multiply writes straight into the trajectory buffer, cuFFT transforms it
// in place and the polar epilogue overwrites each complex sample with its
// (ln|z|, arg z) float2: one buffer of 8 bytes per sample and no extra pass.
#include "common.cuh"
#include "kernels.cuh"

// w = conj(d) / sig2 for both detectors: din = [d_H (nf complex128) | d_L | sig2_H (nf) | sig2_L]
__global__ void k_weights(const double *__restrict__ din, int nf, float2 *__restrict__ w)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= 2 * nf) return;
    const int det = j / nf, f = j - det * nf;
    const double re = din[2 * (det * nf + f)], im = din[2 * (det * nf + f) + 1];
    const double s2 = din[4 * nf + det * nf + f];
    w[j] = make_float2((float)(re / s2), (float)(-im / s2));
}

// one thread per (template, sample): zero outside the band, W * w inside
__global__ void k_premul(const float2 *__restrict__ W, const float2 *__restrict__ w, int nm, int nf, int lo,
                         int nt, float2 *__restrict__ pad)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = 2LL * nm * nt;
    if (idx >= total) return;
    const int det = (int)(idx / ((long long)nm * nt));
    const long long rem = idx - (long long)det * nm * nt;
    const int m = (int)(rem / nt), t = (int)(rem - (long long)m * nt);
    const int f = t - lo;
    float2 o = make_float2(0.f, 0.f);
    if (f >= 0 && f < nf) {
        const float2 a = W[(long long)m * nf + f], b = w[det * nf + f];
        o.x = __fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y));
        o.y = __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x));
    }
    pad[idx] = o;
}

// in place: z -> (ln|z|, arg z)
__global__ void k_polar(float2 *__restrict__ z, long long n)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (; i < n; i += stride) {
        const float2 v = z[i];
        const float p = __fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y));
        z[i] = make_float2(0.5f * logf(fmaxf(p, 1e-38f)), atan2f(v.y, v.x));
    }
}

void exm_run_filter(exm_ctx *ctx, exm_slot &sl, const float2 *dW, int nm)
{
    const int nt = ctx->nt, nf = ctx->nfreq;
    float2 *traj = (float2 *)sl.traj.p;
    float2 *w = (float2 *)((char *)sl.din.p + (size_t)6 * nf * sizeof(double));
    k_weights<<<(2 * nf + 255) / 256, 256, 0, ctx->stream>>>((const double *)sl.din.p, nf, w);
    const long long total = 2LL * nm * nt;
    k_premul<<<(unsigned)((total + 255) / 256), 256, 0, ctx->stream>>>(dW, w, nm, nf, ctx->lo, nt, traj);
    EXM_CUDA(cudaGetLastError());
    exm_fft_plan(ctx, 2 * nm);
    EXM_CUFFT(cufftExecC2C(ctx->plan, (cufftComplex *)traj, (cufftComplex *)traj, CUFFT_FORWARD));
    k_polar<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(traj, total);
    EXM_CUDA(cudaGetLastError());
    ctx->launches += 3;
}
