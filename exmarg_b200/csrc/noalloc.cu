// exm_gather_noalloc: the float64 gather contract (exm_gather) for callers that cannot
// allocate device memory while they call it -- code that runs between the steps of an
// enclosing framework's memory pool, with a budget that is already spent, or from a
// context where an allocation would synchronise the device.  Everything the call reads
// and writes is passed in as device pointers the caller owns; the per-lag partial sums
// the gather needs live in a file-scope device array of fixed size instead of a buffer
// allocated per call.
//
// The array is part of the library image: every device that loads the library holds it
// (16 MiB + 256 B) until the process exits.  Host code must not hand the array's name
// to a kernel (it is a host-side stand-in, not a device address).  With CUDA's lazy
// module loading the array and the kernels of this file would only be loaded -- device
// memory allocated -- on their first use, so exm_ctx_create loads them (exm_noalloc_load):
// it looks the device addresses up with cudaGetSymbolAddress, with the context's device
// current, and queries every kernel of this file.  The addresses are looked up again by
// every context creation on the device (a device reset between contexts gets fresh
// ones); they assume the device's primary context outlives the contexts created on it.
// A call made without a context creation on its device since the process started (not
// possible through this ABI) would look them up itself; make the first call before any
// stream capture.  All calls share the array and it keeps the previous call's contents;
// the error word is cleared at the start of every call, and two calls that overlap on
// the GPU (two contexts or streams at once) race on it.
#include <mutex>

#include "common.cuh"
#include "kernels.cuh"

// (n_slot * n_lag * n_row) at most: 2^20 partial (max, sum) pairs
#define EXM_NOALLOC_MAX_ENTRIES (1 << 20)

static __device__ __align__(256) double g_noalloc_scratch[2 * EXM_NOALLOC_MAX_ENTRIES];
static __device__ __align__(256) unsigned g_noalloc_err[64];

#define EXM_NOALLOC_MAX_DEVICES 64

static std::mutex g_noalloc_mu;
static double *g_noalloc_addr[EXM_NOALLOC_MAX_DEVICES];
static unsigned *g_noalloc_err_addr[EXM_NOALLOC_MAX_DEVICES];

// the device addresses of the scratch array and the error word on device dev (current);
// refresh: look them up again even if known
static void noalloc_addresses(int dev, double **scratch, unsigned **err, bool refresh = false)
{
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (dev < 0 || dev >= EXM_NOALLOC_MAX_DEVICES) EXM_THROW(EXM_ERR_ARG, "device index out of range");
    if (refresh || !g_noalloc_addr[dev]) {
        void *p = nullptr, *q = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            EXM_THROW(EXM_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        e = cudaGetSymbolAddress(&q, g_noalloc_err);
        if (e != cudaSuccess)
            EXM_THROW(EXM_ERR_CUDA, std::string("cudaGetSymbolAddress(error word): ") + cudaGetErrorString(e));
        g_noalloc_addr[dev] = (double *)p;
        g_noalloc_err_addr[dev] = (unsigned *)q;
    }
    *scratch = g_noalloc_addr[dev];
    *err = g_noalloc_err_addr[dev];
}

struct NoAllocArgs {
    const float *lqH, *phH, *lqL, *phL;
    const int32_t *sel;
    const float *lw;
    const int64_t *ids, *tab;
    const double *lna;
    const void *T;              // node tables (element type TE of the kernel)
    const float *tsc;           // per node scale
    const int *tau;
    double *om, *os;
    unsigned *err;
    long long tstride;
    int nm, nt, nwalk, ns, nsel, nn, nphif, nb, nd, ndp, ntau;
    double beta0, dbeta, rph, rdb, rdd, offd;
};

// one block per (row, lag): running (max, sum) over the walked times, float64, per slot
template <typename TE>
__global__ void __launch_bounds__(256) k_gather_noalloc(NoAllocArgs a)
{
    __shared__ double shm[8], shs[8];
    const int j = blockIdx.x, r = blockIdx.y;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long mid = a.ids[j];
    const bool row_ok = mid >= 0 && mid < a.nm;
    if (!row_ok && threadIdx.x == 0) atomicOr(a.err, 1u);
    const int nt = a.nt;
    const int tau0 = ((a.tau[r] % nt) + nt) % nt;
    for (int n = 0; n < a.ns; ++n) {
        const long long tb = a.tab[(long long)j * a.ns + n];
        const bool ok = row_ok && tb >= 0 && tb < a.nn;
        if (!ok && threadIdx.x == 0 && row_ok) atomicOr(a.err, 2u);
        const double offb = (a.lna[(long long)j * a.ns + n] - a.beta0) / a.dbeta;
        double m = -1e300, s = 0.0;
        for (int k = threadIdx.x; ok && k < a.nwalk; k += blockDim.x) {
            const int t = a.sel ? a.sel[mid * a.nwalk + k] : k;
            if (t < 0 || t >= nt) {
                atomicOr(a.err, 4u);
                continue;
            }
            int i1 = t + tau0;
            if (i1 >= nt) i1 -= nt;
            const float2 l = make_float2(a.lqL[mid * nt + t], a.phL[mid * nt + t]);
            const float2 h = make_float2(a.lqH[mid * nt + i1], a.phH[mid * nt + i1]);
            double acc = exm_tap_fp64<TE>(l, h, 0.f, 0.f, offb, r, (const TE *)a.T + tb * a.tstride, a.tsc[tb], a.nphif, a.nb,
                                          a.nd, a.ndp, a.rph, a.rdb, a.rdd, a.offd);
            if (a.sel) acc += (double)a.lw[mid * a.nwalk + k];
            if (acc > m) {
                s = s * exp(m - acc) + 1.0;
                m = acc;
            } else {
                s += exp(acc - m);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double m2 = __shfl_down_sync(0xffffffffu, m, o), s2 = __shfl_down_sync(0xffffffffu, s, o);
            if (m2 > m) {
                s = s2 + s * exp(m - m2);
                m = m2;
            } else {
                s = s + s2 * exp(m2 - m);
            }
        }
        if (lane == 0) {
            shm[warp] = m;
            shs[warp] = s;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double M = shm[0], S = shs[0];
            for (int q = 1; q < (int)(blockDim.x >> 5); ++q) {
                if (shm[q] > M) {
                    S = shs[q] + S * exp(M - shm[q]);
                    M = shm[q];
                } else {
                    S = S + shs[q] * exp(shm[q] - M);
                }
            }
            const long long o = ((long long)n * a.ntau + r) * a.nsel + j;
            a.om[o] = M;
            a.os[o] = S;
        }
        __syncthreads();
    }
}

// log-sum-exp over the lags of the scratch partial sums, minus ln n_time, into the caller's output
__global__ void k_gather_noalloc_lags(const double *__restrict__ om, const double *__restrict__ os, int ns, int ntau,
                                      int nsel, int nt, double *__restrict__ out)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= ns * nsel) return;
    const int n = idx / nsel, j = idx - n * nsel;
    double mx = -INFINITY;
    for (int r = 0; r < ntau; ++r) mx = fmax(mx, om[((long long)n * ntau + r) * nsel + j]);
    double tot = 0.0;
    for (int r = 0; r < ntau; ++r) {
        const long long o = ((long long)n * ntau + r) * nsel + j;
        tot += os[o] * exp(om[o] - mx);
    }
    out[idx] = mx + log(tot) - log((double)nt);
}

// Called by exm_ctx_create with device dev current: loads this file's module (the scratch array) and its
// kernels now, so that exm_gather_noalloc allocates nothing on its first call either.
void exm_noalloc_load(int dev)
{
    double *scratch = nullptr;
    unsigned *err = nullptr;
    noalloc_addresses(dev, &scratch, &err, true);
    cudaFuncAttributes fa;
    EXM_CUDA(cudaFuncGetAttributes(&fa, (const void *)k_gather_noalloc<float>));
    EXM_CUDA(cudaFuncGetAttributes(&fa, (const void *)k_gather_noalloc<__half>));
    EXM_CUDA(cudaFuncGetAttributes(&fa, (const void *)k_gather_noalloc<__nv_bfloat16>));
    EXM_CUDA(cudaFuncGetAttributes(&fa, (const void *)k_gather_noalloc_lags));
}

extern "C" int exm_gather_noalloc(exm_ctx *ctx, int nm, int n_time, const float *lqH, const float *phH,
                                  const float *lqL, const float *phL, int nwalk, const int32_t *sel, const float *lw,
                                  int nsel, int ns, const int64_t *mass_ids, const double *lna, const int64_t *tab_ids,
                                  double *out)
{
    if (!ctx) return EXM_ERR_ARG;
    try {
        EXM_CUDA(cudaSetDevice(ctx->dev));
        if (!ctx->T.p) EXM_THROW(EXM_ERR_STATE, "no store on this context (exm_store_init and its nodes first)");
        if (nm < 1 || n_time < 1 || nsel < 1 || ns < 1 || nwalk < 0)
            EXM_THROW(EXM_ERR_ARG, "need nm, n_time, nsel, ns >= 1 and nwalk >= 0");
        if (!lqH || !phH || !lqL || !phL || !mass_ids || !lna || !tab_ids || !out || (nwalk > 0 && (!sel || !lw)))
            EXM_THROW(EXM_ERR_ARG, "null device pointer");
        const long long entries = (long long)ns * ctx->ntau * nsel;
        if (entries > EXM_NOALLOC_MAX_ENTRIES)
            EXM_THROW(EXM_ERR_ARG, "n_slot * n_lag * n_row = " + std::to_string(entries) +
                                       " exceeds the fixed scratch of exm_gather_noalloc (" +
                                       std::to_string(EXM_NOALLOC_MAX_ENTRIES) + " entries)");
        double *scratch = nullptr;
        unsigned *err = nullptr;
        noalloc_addresses(ctx->dev, &scratch, &err);
        EXM_CUDA(cudaMemsetAsync(err, 0, sizeof(unsigned), ctx->stream));
        NoAllocArgs a;
        a.lqH = lqH;
        a.phH = phH;
        a.lqL = lqL;
        a.phL = phL;
        a.sel = nwalk > 0 ? sel : nullptr;
        a.lw = lw;
        a.ids = mass_ids;
        a.tab = tab_ids;
        a.lna = lna;
        a.T = ctx->T.p;
        a.tsc = (const float *)ctx->d_tscale.p;
        a.tau = (const int *)ctx->d_tau.p;
        a.om = scratch;
        a.os = scratch + EXM_NOALLOC_MAX_ENTRIES;
        a.err = err;
        a.tstride = (long long)ctx->tstride;
        a.nm = nm;
        a.nt = n_time;
        a.nwalk = nwalk > 0 ? nwalk : n_time;
        a.ns = ns;
        a.nsel = nsel;
        a.nn = ctx->nn;
        a.nphif = ctx->nphif;
        a.nb = ctx->nb;
        a.nd = ctx->nd;
        a.ndp = ctx->ndp;
        a.ntau = ctx->ntau;
        a.beta0 = ctx->beta0;
        a.dbeta = ctx->dbeta;
        a.rph = EXM_NPHI / 6.283185307179586;
        a.rdb = 2.0 / ctx->dbeta;
        a.rdd = 1.0 / ctx->ddelta;
        a.offd = -ctx->delta0 / ctx->ddelta;
        dim3 grid(nsel, ctx->ntau);
        if (ctx->dtype == EXM_DTYPE_F16)
            k_gather_noalloc<__half><<<grid, 256, 0, ctx->stream>>>(a);
        else if (ctx->dtype == EXM_DTYPE_BF16)
            k_gather_noalloc<__nv_bfloat16><<<grid, 256, 0, ctx->stream>>>(a);
        else
            k_gather_noalloc<float><<<grid, 256, 0, ctx->stream>>>(a);
        k_gather_noalloc_lags<<<(ns * nsel + 255) / 256, 256, 0, ctx->stream>>>(a.om, a.os, ns, ctx->ntau, nsel, n_time,
                                                                               out);
        EXM_CUDA(cudaGetLastError());
        unsigned e = 0;
        EXM_CUDA(cudaMemcpyAsync(&e, err, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
        EXM_CUDA(cudaStreamSynchronize(ctx->stream));
        if (e & 1u) EXM_THROW(EXM_ERR_ARG, "mass id out of range");
        if (e & 2u) EXM_THROW(EXM_ERR_ARG, "table id out of range");
        if (e & 4u) EXM_THROW(EXM_ERR_ARG, "visited time out of range");
    } catch (const exm_error &e) {
        ctx->err = e.msg;
        return e.code;
    } catch (const std::exception &e) {
        ctx->err = e.what();
        return EXM_ERR_CUDA;
    }
    return EXM_OK;
}
