// Device helpers shared by the kernels, and the host-side launchers of each stage.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>

#include "common.cuh"

// staging window of one (node, lag, phase plane): rows of beta x columns of Delta
#define EXM_WB 80
#define EXM_WD 164     // float32 tables: row pitch = 4 banks mod 32, neighbouring rows start on different banks
#define EXM_WD16 168   // 16-bit tables: a multiple of 8 elements (16-byte TMA rows), pitch 20 banks mod 32

// Table elements as stored: float32, or 16-bit with a per-node scale (value = scale * element;
// the scale is a power of two for float16 and 1 for bfloat16, so the product is exact).
template <typename TE> struct TabElem;
template <> struct TabElem<float> {
    static constexpr int wd = EXM_WD;
    static constexpr int calign = 4;   // window column origin: a multiple of 16 bytes
    static constexpr CUtensorMapDataType tma = CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    __device__ static __forceinline__ float ld(const float *p) { return __ldg(p); }
    __device__ static __forceinline__ float cvt(float v) { return v; }
};
template <> struct TabElem<__half> {
    static constexpr int wd = EXM_WD16;
    static constexpr int calign = 8;
    static constexpr CUtensorMapDataType tma = CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
    __device__ static __forceinline__ float ld(const __half *p) { return __half2float(__ldg(p)); }
    __device__ static __forceinline__ float cvt(__half v) { return __half2float(v); }
};
template <> struct TabElem<__nv_bfloat16> {
    static constexpr int wd = EXM_WD16;
    static constexpr int calign = 8;
    static constexpr CUtensorMapDataType tma = CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    __device__ static __forceinline__ float ld(const __nv_bfloat16 *p) { return __bfloat162float(__ldg(p)); }
    __device__ static __forceinline__ float cvt(__nv_bfloat16 v) { return __bfloat162float(v); }
};

// bytes per stored element, window columns and column alignment of a store dtype (EXM_DTYPE_*)
inline size_t exm_dtype_bytes(int dtype) { return dtype == EXM_DTYPE_F32 ? 4 : 2; }
inline int exm_dtype_wd(int dtype) { return dtype == EXM_DTYPE_F32 ? EXM_WD : EXM_WD16; }
inline int exm_dtype_calign(int dtype) { return dtype == EXM_DTYPE_F32 ? 4 : 8; }
#define EXM_TCH 2048        // templates per gather block

// Tap descriptors of one lag, sorted by (plane pair, template), are stored in chunks of
// EXM_DCH = 32 * EXM_TPL.  The gather's lane l takes the consecutive taps l*TPL .. l*TPL+TPL-1
// of a chunk (so equal templates meet in registers), and they are stored lane-interleaved --
// tap i of lane l at i*32 + l -- so that every load instruction of a warp reads 32 consecutive
// descriptors (512 bytes) instead of 32 scattered cache lines.
#ifndef EXM_TPL
#define EXM_TPL 16
#endif
#define EXM_DCH (32 * EXM_TPL)
static_assert((EXM_TPL & (EXM_TPL - 1)) == 0, "taps per lane must be a power of two");

// storage index of the descriptor at sorted position j (within its lag)
__host__ __device__ __forceinline__ long long exm_desc_phys(long long j)
{
    const long long q = j & (EXM_DCH - 1);
    return (j - q) + (q % EXM_TPL) * 32 + q / EXM_TPL;
}

// descriptors per lag as stored: whole chunks
inline long long exm_desc_pitch(long long per_lag) { return (per_lag + EXM_DCH - 1) / EXM_DCH * EXM_DCH; }
#define EXM_MAX_CHUNK 8192  // templates per pass (13-bit template field of a descriptor)
#define EXM_MAX_NODES 64
#define EXM_HB_LO (-1024)   // beta-hat histogram covers [-1024, 1024)
#define EXM_HB_N 2048

struct TapGeom {
    double rph;   // NPHI / (2 pi)
    double rdb;   // 2 / dbeta
    double rdd;   // 1 / ddelta
    double offd;  // -delta0 / ddelta
    int nd, nt;
};

// The per-tap quantities that do not depend on the node (the reference computes
// them per node, exmarg/search/gather.py:50-82): the plane pair p and the weight w
// of plane p + 1, beta-hat = ln|z_L| 2/dbeta - ln(u)/dbeta as floor + fraction,
// and the Delta coordinate of the unclamped-beta case as (d0, fd).
// ln|z| enters as its float32 value plus the filter's float32 residual (llo, hlo: ln|z| - float(ln|z|), zero for
// trajectories given as float32), so beta-hat and Delta see the filter's float64 value; the phases stay float32
// and are subtracted in float32, as the reference does.
__device__ __forceinline__ void exm_tap_geom(float2 l, float2 h, float llo, float hlo, double boff, const TapGeom &g,
                                             int &p, float &w, int &ib, float &fb, int &d0, float &fd)
{
    double x3 = (double)(h.y - l.y) * g.rph;   // float32 difference, float64 scale, as the reference
    if (x3 < 0.0) x3 += EXM_NPHI;
    if (x3 >= EXM_NPHI) x3 -= EXM_NPHI;
    int c0 = (int)x3;
    c0 = c0 < 0 ? 0 : (c0 > EXM_NPHI - 1 ? EXM_NPHI - 1 : c0);
    const double fc = x3 - c0;
    // planes ci0 = reflect(c0) and ci1 = reflect(c0 + 1) are always {p, p + 1}
    if (c0 <= EXM_NPAIR - 1) {
        p = c0;
        w = (float)fc;
    } else {
        p = EXM_NPHI - 1 - c0;
        w = (float)(1.0 - fc);
    }
    const double aL = (double)l.x + (double)llo, aH = (double)h.x + (double)hlo;
    const double bh = aL * g.rdb + boff;
    const double fl = floor(bh);
    ib = (int)fmax(fmin(fl, 1023.0), -1024.0);
    fb = (float)(bh - fl);
    double xd = (aH - aL) * g.rdd + g.offd;
    if (xd < 0.0) xd = 0.0; else if (xd > g.nd - 1 - 1e-6) xd = g.nd - 1 - 1e-6;
    d0 = (int)xd;
    fd = (float)(xd - d0);
}

// the reference's tap value in float64 (exmarg/search/gather.py:50-93) for one
// node table Tn (padded rows of ndp elements, value = scale * element), lag row r;
// lw added by the caller
template <typename TE>
__device__ __forceinline__ double exm_tap_fp64(float2 l, float2 h, float llo, float hlo, double offb, int r,
                                               const TE *__restrict__ Tn,
                                               float scale, int nphif, int nb, int nd, int ndp, double rph, double rdb,
                                               double rdd, double offd)
{
    double x3 = (double)(h.y - l.y) * rph;
    if (x3 < 0.0) x3 += EXM_NPHI;
    if (x3 >= EXM_NPHI) x3 -= EXM_NPHI;
    int c0 = (int)x3;
    c0 = c0 < 0 ? 0 : (c0 > EXM_NPHI - 1 ? EXM_NPHI - 1 : c0);
    const double fc = x3 - c0;
    const int c1 = (c0 + 1) % EXM_NPHI;
    const double aH = (double)h.x + (double)hlo, aL = (double)l.x + (double)llo;
    const double xbr = aL * rdb + offb;
    double xb = xbr;
    if (xb < 0.0) xb = 0.0; else if (xb > nb - 1 - 1e-6) xb = nb - 1 - 1e-6;
    const double aLc = aL + (xb - xbr) / rdb;
    double xd = (aH - aLc) * rdd + offd;
    if (xd < 0.0) xd = 0.0; else if (xd > nd - 1 - 1e-6) xd = nd - 1 - 1e-6;
    const int d0 = (int)xd;
    const double fdf = xd - d0, fd0 = 1.0 - fdf;
    const int d1 = d0 + 1 < nd ? d0 + 1 : nd - 1;
    const int b0 = (int)xb;
    const double fbf = xb - b0, fb0 = 1.0 - fbf;
    const int b1 = b0 + 1 < nb ? b0 + 1 : nb - 1;
    double acc = 0.0;
#pragma unroll
    for (int cc = 0; cc < 2; ++cc) {
        int ci = cc ? c1 : c0;
        if (ci > EXM_NPHI / 2) ci = EXM_NPHI - ci;
        const double fci = cc ? fc : 1.0 - fc;
        const TE *r0 = Tn + (((long long)r * nphif + ci) * nb + b0) * ndp;
        const TE *r1 = Tn + (((long long)r * nphif + ci) * nb + b1) * ndp;
        const double v = fb0 * (fd0 * (double)TabElem<TE>::ld(r0 + d0) + fdf * (double)TabElem<TE>::ld(r0 + d1)) +
                         fbf * (fd0 * (double)TabElem<TE>::ld(r1 + d0) + fdf * (double)TabElem<TE>::ld(r1 + d1));
        acc += fci * v;
    }
    return acc * (double)scale;
}

// ------------------------------------------------------------------ launchers

void exm_store_quantize(exm_ctx *ctx, int k, const float *src, int sp);
// nodes first..first+n-1 from files (at byte offsets) or host arrays through pinned staging (storeio.cu)
void exm_store_load_run(exm_ctx *ctx, int first, int n, const char *const *paths, const int64_t *offsets,
                        const float *const *hosts, int readers, long long chunk_bytes, int flags, double *stats);
void exm_redshift_release(exm_ctx *ctx);
void exm_store_dequantize(exm_ctx *ctx, int k, float *dst, int dp);

void exm_fft_plan(exm_ctx *ctx, int batch);
void exm_run_filter(exm_ctx *ctx, exm_slot &sl, const float2 *dW, int nm);
void exm_run_pcg(exm_ctx *ctx, exm_slot &sl, const uint64_t *d_state, int K, int S);
void exm_pcg_words(uint64_t seed, uint64_t *w);
void exm_run_topk(exm_ctx *ctx, exm_slot &sl, int nmc, const int *d_order_chunk, int K, int S);

struct ChunkInfo {
    int m_base;   // first internal template of the chunk
    int nmc;      // templates in the chunk
    int nwalk;    // walked times per template (n_time when every time is walked)
    int use_sel;  // sel holds the walked times
    float lw;     // log weight of a random draw
};
void exm_run_taps(exm_ctx *ctx, exm_slot &sl, const ChunkInfo &ci, int r0, int rc, bool first_chunk_of_lags);
void exm_run_gather_planes(exm_ctx *ctx, exm_slot &sl, const ChunkInfo &ci, int r0, int rc);
int exm_gather_num_cfgs();
void exm_run_node_lse(exm_ctx *ctx, exm_slot &sl, int m_base, int nmc);
void exm_run_lnb(exm_ctx *ctx, exm_slot &sl);
void exm_run_gather_simple(exm_ctx *ctx, exm_slot &sl, int nsel, int ns, const int *d_rows, const int *d_tab,
                           const double *d_lna, int nwalk, int use_sel, float lw, double *d_out);
void exm_run_distance_weights(exm_ctx *ctx, double ymin, int prior, const double *d_lny, const double *d_p,
                              int n_dens);
