// Resident tables.  The node tables T[k][tau][phi+][beta][Delta] live in one device
// allocation with each Delta row padded from nd to ndp floats (a multiple of 4,
// so every row starts on a 16-byte boundary as the TMA tensor map requires).
// Replaces exmarg/search/store.py:204-214 (upload): the tables are copied once and
// stay resident for every call.
#include <cudaTypedefs.h>

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
    const cuuint64_t row = (cuuint64_t)ctx->ndp * 4;
    cuuint64_t strides[4] = {row, row * ctx->nb, row * ctx->nb * ctx->nphif, row * ctx->nb * ctx->nphif * ctx->ntau};
    cuuint32_t box[5] = {EXM_WD, EXM_WB, 1, 1, 1};
    cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    CUresult r = get_encode()(&ctx->tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, ctx->T.p, dims, strides, box, estr,
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
    float *Tk = (float *)ctx->T.p + (size_t)k * ctx->tstride;
    k_generate_node<<<ctx->sm_count * 16, 256, 0, ctx->stream>>>(Tk, dM, dP, dQ, S, seed, (uint32_t)k, ctx->ntau,
                                                                ctx->nphif, ctx->nb, ctx->nd, ctx->ndp);
    EXM_CUDA(cudaGetLastError());
    EXM_CUDA(cudaStreamSynchronize(ctx->stream));
    exm_free(ctx, tmp);
}
