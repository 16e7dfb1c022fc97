// Matched filter of one segment against the whole bank (exmarg/search/bank.py:56-78):
//   w_I = complex64(conj(d_I) / sig2_I)          (float64 division, rounded once)
//   pad[m, lo:lo+nf] = W[m] * w_I                 (complex64 product, no FMA contraction)
//   z = FFT_forward(pad)                          (cuFFT Z2Z, length n_time, batched)
//   (ln|z|, arg z) = (0.5 ln max(re^2 + im^2, 1e-38), atan2(im, re)), rounded once to float32 as the
//   reference rounds them; with filter precision 'fp64' also the float32 residual ln|z| - float(ln|z|), which
//   the tap geometry adds back (the float32 rounding of ln|z| moves loud taps by ~1e-5 in ln Lambda through the
//   table slopes, in the reference as here)
// The complex64 product (the reference's pad) is transformed in float64, so each
// trajectory sample is the float32 rounding of the exact filter output of that pad:
// a float32 FFT adds its own rounding (cuFFT's is several times larger than numpy's),
// which the table slopes amplify into ln Lambda.  The pre-multiply writes the padded
// rows straight into the FFT buffer, cuFFT transforms them in place, and the polar
// epilogue writes (ln|z|, arg z) float2 pairs into the trajectory buffer.
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

// one thread per (template, sample): zero outside the band, W * w inside (complex64 product)
__global__ void k_premul(const float2 *__restrict__ W, const float2 *__restrict__ w, int nm, int nf, int lo,
                         int nt, double2 *__restrict__ pad)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = 2LL * nm * nt;
    if (idx >= total) return;
    const int det = (int)(idx / ((long long)nm * nt));
    const long long rem = idx - (long long)det * nm * nt;
    const int m = (int)(rem / nt), t = (int)(rem - (long long)m * nt);
    const int f = t - lo;
    double2 o = make_double2(0.0, 0.0);
    if (f >= 0 && f < nf) {
        const float2 a = W[(long long)m * nf + f], b = w[det * nf + f];
        o.x = (double)__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y));
        o.y = (double)__fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x));
    }
    pad[idx] = o;
}

// z (float64) -> (ln|z|, arg z) float32 and, if lo is not null, the residual of ln|z|
__global__ void k_polar(const double2 *__restrict__ z, float2 *__restrict__ out, float *__restrict__ lo, long long n)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (; i < n; i += stride) {
        const double2 v = z[i];
        const double p = v.x * v.x + v.y * v.y;
        const double lq = 0.5 * log(fmax(p, 1e-38));
        const float hi = (float)lq;
        out[i] = make_float2(hi, (float)atan2(v.y, v.x));
        if (lo) lo[i] = (float)(lq - (double)hi);
    }
}

void exm_run_filter(exm_ctx *ctx, exm_slot &sl, const float2 *dW, int nm)
{
    const int nt = ctx->nt, nf = ctx->nfreq;
    float2 *traj = (float2 *)sl.traj.p;
    float2 *w = (float2 *)((char *)sl.din.p + (size_t)6 * nf * sizeof(double) + 4 * sizeof(uint64_t));
    k_weights<<<(2 * nf + 255) / 256, 256, 0, ctx->stream>>>((const double *)sl.din.p, nf, w);
    const long long total = 2LL * nm * nt;
    double2 *z = (double2 *)sl.fft.p;
    k_premul<<<(unsigned)((total + 255) / 256), 256, 0, ctx->stream>>>(dW, w, nm, nf, ctx->lo, nt, z);
    EXM_CUDA(cudaGetLastError());
    exm_fft_plan(ctx, 2 * nm);
    EXM_CUFFT(cufftExecZ2Z(ctx->plan, (cufftDoubleComplex *)z, (cufftDoubleComplex *)z, CUFFT_FORWARD));
    k_polar<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(z, traj, ctx->traj_fp64 ? (float *)sl.trajlo.p : nullptr,
                                                         total);
    EXM_CUDA(cudaGetLastError());
    ctx->launches += 3;
}
