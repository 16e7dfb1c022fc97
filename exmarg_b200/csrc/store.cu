// Resident tables.  The node tables T[k][tau][phi+][beta][Delta] live in one device
// allocation with each Delta row padded from nd to ndp elements (16 bytes a row, as
// the TMA tensor map requires).  Elements are float32, or float16 / bfloat16 with a
// per-node scale (value = scale * element): float16 uses the power of two that puts
// the node's largest |value| just below 2^15 (so scaling is exact and the range
// fits), bfloat16 has float32's range and a scale of 1.  Both round to nearest even.
// Replaces exmarg/search/store.py:110-120 (upload): the tables are copied once and
// stay resident for every call.
#include <cudaTypedefs.h>

#include <cmath>
#include <cstring>

#include "common.cuh"
#include "kernels.cuh"

// ------------------------------------------------------------------ seeded synthetic tables

__device__ __forceinline__ uint32_t mix32(uint32_t h)
{
    h ^= h >> 16;
    h *= 0x7FEB352Du;
    h ^= h >> 15;
    h *= 0x846CA68Bu;
    return h ^ (h >> 16);
}

// the same float32 operations, in the same order, as exmarg_b200.synth.gen_table_node
__global__ void k_generate_node(float *__restrict__ Tk, const float *__restrict__ M, const float *__restrict__ P,
                                const float *__restrict__ Q, float S, uint32_t seed, uint32_t k, int ntau, int nphif,
                                int nb, int nd, int ndp)
{
    const long long n = (long long)ntau * nphif * nb * ndp;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (; idx < n; idx += stride) {
        const int d = (int)(idx % ndp);
        long long rest = idx / ndp;
        const int b = (int)(rest % nb);
        rest /= nb;
        const int c = (int)(rest % nphif);
        const int r = (int)(rest / nphif);
        if (d >= nd) {
            Tk[idx] = 0.f;
            continue;
        }
        float v = __fmul_rn(M[b * nd + d], P[c]);
        v = __fmul_rn(v, Q[r]);
        v = __fsub_rn(v, S);
        uint32_t h = (seed * 0x9E3779B1u) ^ (k * 0x85EBCA77u);
        h = mix32(h ^ ((uint32_t)r * 0xC2B2AE3Du));
        h = mix32(h ^ ((uint32_t)c * 0x27D4EB2Fu));
        h = mix32(h ^ ((uint32_t)b * 0x165667B1u));
        h = mix32(h ^ ((uint32_t)d * 0xD3A2646Cu));
        const float pert = (float)((int)(h & 0xFFFFu) - 32768) * 2.384185791015625e-07f;   // 2^-22
        Tk[idx] = __fadd_rn(v, pert);
    }
}

// ------------------------------------------------------------------ 16-bit storage

// largest |value| of n floats (as ordered bits of a non-negative float)
__global__ void k_absmax(const float *__restrict__ x, long long n, unsigned *out)
{
    float m = 0.f;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(x[i]));
    m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 16));
    m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 8));
    m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 4));
    m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 2));
    m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 1));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

template <typename TE> __device__ __forceinline__ TE to_elem(float v);
template <> __device__ __forceinline__ __half to_elem<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 to_elem<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

// rows of nd values (source pitch sp) -> elements round(v * inv_scale) (pitch dp, padding zero)
template <typename TE>
__global__ void k_quantize(const float *__restrict__ src, long long rows, int nd, int sp, TE *__restrict__ dst, int dp,
                           float inv_scale)
{
    const long long n = rows * dp;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long row = i / dp;
        const int d = (int)(i - row * dp);
        dst[i] = to_elem<TE>(d < nd ? __fmul_rn(src[row * sp + d], inv_scale) : 0.f);
    }
}

// elements -> float32 values scale * element, rows of nd (pitch sp -> pitch dp)
template <typename TE>
__global__ void k_dequantize(const TE *__restrict__ src, long long rows, int nd, int sp, float *__restrict__ dst, int dp,
                             float scale)
{
    const long long n = rows * nd;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long row = i / nd;
        const int d = (int)(i - row * nd);
        dst[row * dp + d] = __fmul_rn(TabElem<TE>::cvt(src[row * sp + d]), scale);
    }
}

// the float16 scale of a node whose largest |value| is amax: the power of two 2^e with
// amax / 2^e in [2^14, 2^15) (1 for an all-zero node)
static float f16_scale(float amax)
{
    if (!(amax > 0.f)) return 1.f;
    int e = 0;
    (void)std::frexp(amax, &e);   // amax = f 2^e, f in [0.5, 1)
    return std::ldexp(1.f, e - 15);
}

// node k of a 16-bit store from float32 rows already on the device (pitch sp)
void exm_store_quantize(exm_ctx *ctx, int k, const float *src, int sp)
{
    const long long rows = (long long)ctx->ntau * ctx->nphif * ctx->nb;
    float scale = 1.f;
    if (ctx->dtype == EXM_DTYPE_F16) {
        dbuf mx;
        exm_alloc(ctx, mx, sizeof(unsigned));
        EXM_CUDA(cudaMemsetAsync(mx.p, 0, sizeof(unsigned), ctx->stream));
        k_absmax<<<ctx->sm_count * 8, 256, 0, ctx->stream>>>(src, rows * sp, (unsigned *)mx.p);
        EXM_CUDA(cudaGetLastError());
        unsigned bits = 0;
        EXM_CUDA(cudaMemcpyAsync(&bits, mx.p, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
        EXM_CUDA(cudaStreamSynchronize(ctx->stream));
        exm_free(ctx, mx);
        float amax;
        memcpy(&amax, &bits, sizeof(float));
        if (!std::isfinite(amax)) EXM_THROW(EXM_ERR_ARG, "node table holds a non-finite value");
        scale = f16_scale(amax);
        __half *dst = (__half *)ctx->T.p + (size_t)k * ctx->tstride;
        k_quantize<__half><<<ctx->sm_count * 16, 256, 0, ctx->stream>>>(src, rows, ctx->nd, sp, dst, ctx->ndp,
                                                                        1.f / scale);
    } else {
        __nv_bfloat16 *dst = (__nv_bfloat16 *)ctx->T.p + (size_t)k * ctx->tstride;
        k_quantize<__nv_bfloat16><<<ctx->sm_count * 16, 256, 0, ctx->stream>>>(src, rows, ctx->nd, sp, dst, ctx->ndp,
                                                                               1.f);
    }
    EXM_CUDA(cudaGetLastError());
    ctx->tscale[k] = scale;
    EXM_CUDA(cudaMemcpyAsync((float *)ctx->d_tscale.p + k, &ctx->tscale[k], sizeof(float), cudaMemcpyHostToDevice,
                             ctx->stream));
    EXM_CUDA(cudaStreamSynchronize(ctx->stream));
}

// node k as float32 values (scale * element) into device rows of pitch dp
void exm_store_dequantize(exm_ctx *ctx, int k, float *dst, int dp)
{
    const long long rows = (long long)ctx->ntau * ctx->nphif * ctx->nb;
    if (ctx->dtype == EXM_DTYPE_F16)
        k_dequantize<__half><<<ctx->sm_count * 16, 256, 0, ctx->stream>>>(
            (const __half *)ctx->T.p + (size_t)k * ctx->tstride, rows, ctx->nd, ctx->ndp, dst, dp, ctx->tscale[k]);
    else
        k_dequantize<__nv_bfloat16><<<ctx->sm_count * 16, 256, 0, ctx->stream>>>(
            (const __nv_bfloat16 *)ctx->T.p + (size_t)k * ctx->tstride, rows, ctx->nd, ctx->ndp, dst, dp,
            ctx->tscale[k]);
    EXM_CUDA(cudaGetLastError());
}

// ------------------------------------------------------------------ tensor map

static PFN_cuTensorMapEncodeTiled_v12000 get_encode()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        EXM_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !p) EXM_THROW(EXM_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
        fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

void exm_make_tmap(exm_ctx *ctx)
{
    // dims innermost first: Delta (ndp), beta (nb), phase plane (nphif), lag (ntau), node (nn)
    cuuint64_t dims[5] = {(cuuint64_t)ctx->ndp, (cuuint64_t)ctx->nb, (cuuint64_t)ctx->nphif, (cuuint64_t)ctx->ntau,
                          (cuuint64_t)ctx->nn};
    const cuuint64_t row = (cuuint64_t)ctx->ndp * exm_dtype_bytes(ctx->dtype);
    cuuint64_t strides[4] = {row, row * ctx->nb, row * ctx->nb * ctx->nphif, row * ctx->nb * ctx->nphif * ctx->ntau};
    cuuint32_t box[5] = {(cuuint32_t)exm_dtype_wd(ctx->dtype), EXM_WB, 1, 1, 1};
    cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    const CUtensorMapDataType ty = ctx->dtype == EXM_DTYPE_F32   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                   : ctx->dtype == EXM_DTYPE_F16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                                                 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    CUresult r = get_encode()(&ctx->tmap, ty, 5, ctx->T.p, dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) EXM_THROW(EXM_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    ctx->tmap_ok = true;
}

void exm_store_generate(exm_ctx *ctx, int k, const float *M, const float *P, const float *Q, float S, uint32_t seed)
{
    dbuf tmp;
    const size_t nM = (size_t)ctx->nb * ctx->nd;
    exm_alloc(ctx, tmp, sizeof(float) * (nM + ctx->nphif + ctx->ntau));
    float *dM = (float *)tmp.p, *dP = dM + nM, *dQ = dP + ctx->nphif;
    EXM_CUDA(cudaMemcpyAsync(dM, M, sizeof(float) * nM, cudaMemcpyHostToDevice, ctx->stream));
    EXM_CUDA(cudaMemcpyAsync(dP, P, sizeof(float) * ctx->nphif, cudaMemcpyHostToDevice, ctx->stream));
    EXM_CUDA(cudaMemcpyAsync(dQ, Q, sizeof(float) * ctx->ntau, cudaMemcpyHostToDevice, ctx->stream));
    if (ctx->dtype == EXM_DTYPE_F32) {
        float *Tk = (float *)ctx->T.p + (size_t)k * ctx->tstride;
        k_generate_node<<<ctx->sm_count * 16, 256, 0, ctx->stream>>>(Tk, dM, dP, dQ, S, seed, (uint32_t)k, ctx->ntau,
                                                                    ctx->nphif, ctx->nb, ctx->nd, ctx->ndp);
        EXM_CUDA(cudaGetLastError());
    } else {   // float32 values into a scratch node, then quantized
        dbuf f;
        const int sp = (ctx->nd + 3) & ~3;
        exm_alloc(ctx, f, sizeof(float) * (size_t)ctx->ntau * ctx->nphif * ctx->nb * sp);
        k_generate_node<<<ctx->sm_count * 16, 256, 0, ctx->stream>>>((float *)f.p, dM, dP, dQ, S, seed, (uint32_t)k,
                                                                    ctx->ntau, ctx->nphif, ctx->nb, ctx->nd, sp);
        EXM_CUDA(cudaGetLastError());
        exm_store_quantize(ctx, k, (const float *)f.p, sp);
        exm_free(ctx, f);
    }
    EXM_CUDA(cudaStreamSynchronize(ctx->stream));
    exm_free(ctx, tmp);
}
