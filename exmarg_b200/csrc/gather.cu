// The table read of Eq. (C7) (exmarg/search/gather.py:32-107) on the B200.
//
// k_gather_planes (the pe_intrinsic path): one block per (node k, lag r, block of up
// to 2048 templates).  The block walks the 48 phase-plane pairs (p, p+1) of the
// node's lag slab T[k, r]; for each plane it stages, with one TMA copy, a window of
// 80 beta rows x 160 Delta columns into shared memory (three slots: two planes in
// use, one in flight).  The descriptors of the lag are sorted by (plane pair,
// template), and each warp owns a contiguous range of templates, so for each pair a
// warp reads one contiguous run of 16-byte descriptors, evaluates the bilinear x
// linear interpolation from shared memory, and merges the log-sum-exp of each
// template with warp shuffles into a per-template accumulator that only it writes.
// Values are carried as (B, e) with B a stored float32 table value and e a small
// float32 correction, so a tap of size ~1e3 keeps ~1e-7 absolute precision.  Taps
// outside the window, and taps whose beta is clamped to the table, take an exact
// float64 path that reads the table from global memory.
//
// k_gather_simple (the gather_cpu / gather_gpu contract, any table per slot): one
// block per (row, lag), the reference's arithmetic in float64.
#include <type_traits>

#include "common.cuh"
#include "kernels.cuh"

// the plane gather's dynamic shared memory; its parts are addressed by 32-bit byte offsets (fewer
// registers in the tap loop than 64-bit generic pointers)
extern __shared__ __align__(1024) unsigned char exm_gsm[];
__device__ __forceinline__ float *gsm_f(unsigned off) { return (float *)(exm_gsm + off); }

// one staged (node, lag, plane) window of element type TE: EXM_WB rows x TabElem<TE>::wd columns
template <typename TE> __host__ __device__ constexpr int slot_elems() { return EXM_WB * TabElem<TE>::wd; }
template <typename TE> __host__ __device__ constexpr unsigned slot_bytes() { return (unsigned)(slot_elems<TE>() * sizeof(TE)); }
static_assert(slot_bytes<float>() % 128 == 0 && slot_bytes<__half>() % 128 == 0, "slots keep 128-byte alignment");
#define EXM_WAIT_CYCLES (2000000000LL)   // about one second at 1.9 GHz
#define EXM_TEST_WAIT_CYCLES (20000LL)   // the wait-expiry test's limit (no copy is ever in flight then)

struct PlaneArgs {
    const uint4 *desc;
    const int32_t *tside;
    const int *off;
    const float2 *H, *L;
    const float *Hlo, *Llo;      // residuals of ln|z| (filter precision 'fp64'), else null
    const void *T;               // node tables, element type of the kernel's TE
    const int *mlo, *mhi, *bnode, *win, *tau;
    const double *boff, *cb, *ckd;
    double *part;
    unsigned *err;
    unsigned long long *stats;   // [0] slow-path taps, [1] boundary taps (may be null)
    long long tstride, per_lag;
    int nn, ntau, nphif, nb, nd, ndp, nt, nmc, m_base, nm_total, r0, tch, nch;
    float lw;
    double rph, rdb, rdd, offd;
    long long wait_cycles;       // limit of the pipeline's barrier waits (EXM_WAIT_CYCLES)
    int stage;                   // 1: stage the planes; 0 (the wait-expiry test): no copy is issued, so the
                                 // first wait runs out and the kernel returns its timeout status
    int cki[EXM_MAX_NODES];
    float ckf[EXM_MAX_NODES];
    float tsc[EXM_MAX_NODES];    // per node: value = tsc * stored element
};

// ------------------------------------------------------------------ TMA + mbarrier

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void tma_load_plane(const CUtensorMap *map, uint64_t *bar, void *dst, int x, int y, int z,
                                               int w, int v, unsigned bytes)
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], "
        "[%7];" ::"r"(smem_u32(dst)),
        "l"((unsigned long long)map), "r"(x), "r"(y), "r"(z), "r"(w), "r"(v), "r"(smem_u32(bar))
        : "memory");
}


// bounded wait on a phase of an mbarrier; false (and the error word set) if it ran out after `limit` cycles
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, unsigned *err,
                                          long long limit = EXM_WAIT_CYCLES)
{
    const uint32_t a = smem_u32(bar);
    const long long t0 = clock64();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > limit) {
            atomicOr(err, EXM_DEVERR_TIMEOUT);
            return false;
        }
    }
}

// ------------------------------------------------------------------ log-sum-exp of (B, e) values

__device__ __forceinline__ void lse_merge(float &B, float &E, float &S, float B2, float E2, float S2)
{
    // (B, E, S) += (B2, E2, S2): the larger of the two values becomes the reference, without a branch
    const float d = (B2 - B) + (E2 - E);
    const bool up = d > 0.f;
    const float e = __expf(-fabsf(d));
    const float s_up = fmaf(S, e, S2), s_dn = fmaf(S2, e, S);
    B = up ? B2 : B;
    E = up ? E2 : E;
    S = up ? s_up : s_dn;
}

// segmented reduction over lanes with equal id (ids non-decreasing along the lanes of a run);
// afterwards the first lane of each run holds the run's total
__device__ __forceinline__ bool seg_reduce(int id, float &B, float &E, float &S)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int id2 = __shfl_down_sync(0xffffffffu, id, o);
        const float B2 = __shfl_down_sync(0xffffffffu, B, o);
        const float E2 = __shfl_down_sync(0xffffffffu, E, o);
        const float S2 = __shfl_down_sync(0xffffffffu, S, o);
        if (lane + o < 32 && id2 == id) lse_merge(B, E, S, B2, E2, S2);
    }
    const int prev = __shfl_up_sync(0xffffffffu, id, 1);
    return lane == 0 || prev != id;
}

// bilinear in (beta, Delta) on planes p and p+1 of the staged windows, linear in phase;
// value = t00 + eps with t00 the stored value at (p, b0, d0).  16-bit elements are
// interpolated as stored (float32 arithmetic) and the result scaled by the node's power-of-two
// scale, which is exact.
template <typename TE>
__device__ __forceinline__ void interp_window(const TE *s0, const TE *s1, int o, float fbf, float fd, float w, float sc,
                                              float &B, float &E)
{
    constexpr int WD = TabElem<TE>::wd;
    const float t00 = TabElem<TE>::cvt(s0[o]), t01 = TabElem<TE>::cvt(s0[o + 1]);
    const float t10 = TabElem<TE>::cvt(s0[o + WD]), t11 = TabElem<TE>::cvt(s0[o + WD + 1]);
    const float u00 = TabElem<TE>::cvt(s1[o]), u01 = TabElem<TE>::cvt(s1[o + 1]);
    const float u10 = TabElem<TE>::cvt(s1[o + WD]), u11 = TabElem<TE>::cvt(s1[o + WD + 1]);
    const float a0 = t01 - t00, c0 = t10 - t00, e0 = (t11 - t10) - a0;
    const float eps0 = fmaf(fd, a0, fbf * fmaf(fd, e0, c0));
    const float a1 = u01 - u00, c1 = u10 - u00, e1 = (u11 - u10) - a1;
    const float eps1 = fmaf(fd, a1, fbf * fmaf(fd, e1, c1));
    B = t00;
    E = fmaf(w, (u00 - t00) + (eps1 - eps0), eps0);
    if (!std::is_same<TE, float>::value) {
        B *= sc;
        E *= sc;
    }
}

__device__ __forceinline__ void split_double(double v, float &B, float &E)
{
    B = (float)v;
    E = (float)(v - (double)B);
}

// One run of tap descriptors (sorted by template) on the two staged planes of pair p.
// Each lane takes 4 consecutive taps of a 128-tap chunk and merges equal-template taps in
// registers; a template that lies inside one lane's taps is merged into its accumulator by
// that lane, one that spans lanes is combined by a segmented shuffle reduction once per chunk.
// byte offsets below are into exm_gsm
struct RunCtx {
    const uint4 *descr;
    const int32_t *tsr;
    unsigned s0, s1;            // the staged windows of planes p and p + 1 (element type TE)
    float sc;                   // the node's scale (16-bit tables)
    unsigned acc, accst;        // accumulator set of the run's templates (B at acc + 4 (t - lo); E, S at
                                // + accst, + 2 accst)
    unsigned bsh, bcf;          // boundary runs: per-template window-row shift (int; EXM_BSH_NONE for templates
                                // whose boundary point is not this node) and beta fraction
    int lo, m_base, n, k, r;
    int sh;                     // window row of a tap = rb0 + carry + sh (regular runs)
    int up, edge;               // fast path: row <= up, and not (row == edge with beta at the clamp)
    float ckf, lw;
    int tF, tL;                 // the templates at the two ends of this warp's taps (may be shared with
    unsigned eF, eL;            // neighbouring warps): their partials go to this warp's edge slots (B, E, S)
    unsigned q, qn;             // this warp's queue of exact-path taps for the pair (int2 entries) and its count
};

__device__ __forceinline__ void acc_merge(const RunCtx &c, int tr, float B, float E, float S)
{
    const bool f = tr == c.tF, l = tr == c.tL;
    const unsigned off = f ? c.eF : (l ? c.eL : c.acc + 4u * (unsigned)tr);
    const unsigned st = (f || l) ? 4u : c.accst;
    float *pB = gsm_f(off), *pE = gsm_f(off + st), *pS = gsm_f(off + 2 * st);
    float b = *pB, e = *pE, s = *pS;
    lse_merge(b, e, s, B, E, S);
    *pB = b;
    *pE = e;
    *pS = s;
}

#define TPL EXM_TPL   // consecutive taps per lane (in groups of GRP); a warp chunk is EXM_DCH taps
#ifndef EXM_GUNROLL
#define EXM_GUNROLL 2
#endif
constexpr int kGroupUnroll = EXM_GUNROLL;   // tap groups of a chunk unrolled in the lane loop
#define EXM_SLOWQ 8   // exact-path taps a consumer warp queues per plane pair for the producer
#define EXM_BSH_NONE (-(1 << 28))   // bsh entry of a template whose boundary point is another node


// the lane-local running segmented merge of one value (taps arrive sorted by template)
__device__ __forceinline__ void lane_merge(const RunCtx &c, int t, float vB, float vE, float wt, int &cT, float &cB,
                                           float &cE, float &cS, int &fT, float &fB, float &fE, float &fS)
{
    // branch-free except for the rare template that opens and closes inside one lane
    const bool nw = t != cT;
    const bool close = nw && cT >= 0;      // cT closes here
    const bool toF = close && fT < 0;      // ... as the lane's first closed partial
    if (close && !toF) acc_merge(c, cT, cB, cE, cS);
    fT = toF ? cT : fT;
    fB = toF ? cB : fB;
    fE = toF ? cE : fE;
    fS = toF ? cS : fS;
    cT = nw ? t : cT;                      // a new template starts from an empty partial
    cB = nw ? -1e30f : cB;
    cE = nw ? 0.f : cE;
    cS = nw ? 0.f : cS;
    lse_merge(cB, cE, cS, vB, vE, wt);
}

// the exact float64 value of a tap outside the staged window (rare)
#ifndef EXM_SLOW_INLINE
#define EXM_SLOW_INLINE __forceinline__
#endif
template <bool BND, typename TE>
__device__ EXM_SLOW_INLINE double slow_tap(const PlaneArgs &a, int il, int tm, int k, int r, int m_base, float sc)
{
    const int nt = a.nt;
    const int tau0 = ((a.tau[r] % nt) + nt) % nt;
    int i1 = tm + tau0;
    if (i1 >= nt) i1 -= nt;
    const int gi = il + m_base;
    const double offb = (BND ? a.cb[gi] : a.ckd[k]) + a.boff[gi];   // ckd: (ln s_k - beta0)/dbeta
    return exm_tap_fp64<TE>(a.L[(long long)il * nt + tm], a.H[(long long)il * nt + i1],
                            a.Llo ? a.Llo[(long long)il * nt + tm] : 0.f, a.Hlo ? a.Hlo[(long long)il * nt + i1] : 0.f,
                            offb, r,
                            (const TE *)a.T + (long long)k * a.tstride, sc, a.nphif, a.nb, a.nd, a.ndp, a.rph, a.rdb,
                            a.rdd, a.offd);
}

// GRP taps: decode, window interpolation for all of them (no branch between the shared loads),
// the exact float64 value for the rare taps outside the window, then the merges
template <bool BND, int GRP, typename TE>
__device__ __forceinline__ void tap_group(const PlaneArgs &a, const RunCtx &c, const uint4 *q, int j, int pj, int beg,
                                          int end, int &cT, float &cB, float &cE, float &cS, int &fT, float &fB,
                                          float &fE, float &fS, unsigned &n_slow)
{
    // j: sorted position of the group's first tap (taps j .. j + GRP - 1 of this lane);
    // pj: its storage index (tap u of the group at pj + 32 u)
    int t[GRP], o[GRP];
    bool fast[GRP];
    float fbf[GRP], fd[GRP], w[GRP], lwv[GRP], vB[GRP], vE[GRP];
#pragma unroll
    for (int u = 0; u < GRP; ++u) {
        int tt = (j + u >= beg && j + u < end) ? (int)(q[u].w >> 19) + c.m_base - c.lo : -1;
        if (tt >= c.n) {   // outside the block's templates: report and skip
            atomicOr(a.err, EXM_DEVERR_BOUNDS);
            tt = -1;
        }
        // boundary runs: the template's window-row shift, EXM_BSH_NONE unless its boundary point is this node
        int bs = 0;
        if (BND) {
            bs = tt >= 0 ? ((const int *)gsm_f(c.bsh))[tt] : EXM_BSH_NONE;
            if (bs == EXM_BSH_NONE) tt = -1;
        }
        t[u] = tt;
        const int ts = tt >= 0 ? tt : 0;
        const float fb = __uint_as_float(q[u].x);
        fd[u] = __uint_as_float(q[u].y);
        w[u] = __uint_as_float(q[u].z & 0x7FFFFFFFu);
        lwv[u] = (q[u].z >> 31) ? c.lw : 0.f;
        const int rd = (int)((q[u].w >> 11) & 0xFFu);      // window column (255: outside)
        const int rb0 = ((int)(q[u].w << 21)) >> 21;        // beta-hat row from the window origin
        const float sfr = fb + (BND ? gsm_f(c.bcf)[ts] : c.ckf);
        const int cy = sfr >= 1.f;
        fbf[u] = cy ? sfr - 1.f : sfr;
        const int rb = rb0 + cy + (BND ? bs : c.sh);   // this node's window row
        constexpr int WD = TabElem<TE>::wd;
        fast[u] = (unsigned)rb <= (unsigned)c.up && rd <= WD - 2 && !(rb == c.edge && fbf[u] > 0.999999f);
        o[u] = fast[u] ? rb * WD + rd : 0;
    }
#pragma unroll
    for (int u = 0; u < GRP; ++u)
        interp_window<TE>((const TE *)(exm_gsm + c.s0), (const TE *)(exm_gsm + c.s1), o[u], fbf[u], fd[u], w[u], c.sc,
                          vB[u], vE[u]);
    float wt[GRP];
#pragma unroll
    for (int u = 0; u < GRP; ++u) {
        const bool sl = t[u] >= 0 && !fast[u];
        wt[u] = t[u] >= 0 ? 1.f : 0.f;
        if (__any_sync(0xffffffffu, sl)) {
            // exact-path taps go to the warp's queue: the producer computes them 32 at a time instead
            // of stalling the warp on one lane's float64 path; a full queue computes them here
            const int lane = threadIdx.x & 31;
            const unsigned m = __ballot_sync(0xffffffffu, sl);
            int *qn = (int *)(exm_gsm + c.qn);
            const int n0 = *qn;
            const int pos = n0 + __popc(m & ((1u << lane) - 1u));
            __syncwarp();
            if (sl) {
                ++n_slow;
                if (pos < EXM_SLOWQ) {
                    ((int2 *)(exm_gsm + c.q))[pos] =
                        make_int2(pj + 32 * u, (int)(q[u].w >> 19) | (BND ? 1 << 30 : 0) | (int)((q[u].z >> 31) << 29));
                    vB[u] = -1e30f;
                    vE[u] = 0.f;
                    wt[u] = 0.f;
                    lwv[u] = 0.f;
                } else {
                    const double v =
                        slow_tap<BND, TE>(a, (int)(q[u].w >> 19), c.tsr[pj + 32 * u], c.k, c.r, c.m_base, c.sc);
                    split_double(v, vB[u], vE[u]);
                }
            }
            if (lane == 0) *qn = min(EXM_SLOWQ, n0 + __popc(m));
            __syncwarp();
        }
    }
#pragma unroll
    for (int u = 0; u < GRP; ++u)
        lane_merge(c, t[u], vB[u], vE[u] + lwv[u], wt[u], cT, cB, cE, cS, fT, fB, fE, fS);
}

template <bool BND, int GRP, typename TE>
__device__ void process_run(const PlaneArgs &a, const RunCtx &c, int beg, int end, unsigned &n_slow)
{
    // the warp's sorted positions [beg, end), walked in whole chunks of EXM_DCH (positions outside
    // [beg, end) masked); lane l takes the chunk's positions l*TPL + i, stored at i*32 + l
    const int lane = threadIdx.x & 31;
    const int jstart = beg & ~(EXM_DCH - 1);
    uint4 qa[GRP];
#pragma unroll
    for (int u = 0; u < GRP; ++u) {
        const int jl = jstart + TPL * lane + u;
        qa[u] = (jl >= beg && jl < end) ? __ldg(c.descr + jstart + 32 * u + lane) : make_uint4(0u, 0u, 0u, 0u);
    }
    for (int j0 = jstart; j0 < end; j0 += EXM_DCH) {
        const int jb = j0 + TPL * lane;
        int cT = -1, fT = -1;
        float cB = -1e30f, cE = 0.f, cS = 0.f, fB = -1e30f, fE = 0.f, fS = 0.f;
#pragma unroll(kGroupUnroll)
        for (int g = 0; g < TPL / GRP; ++g) {
            uint4 cur[GRP];
#pragma unroll
            for (int u = 0; u < GRP; ++u) cur[u] = qa[u];
            // the next group of descriptors (this lane's next group, or the next chunk's first)
            const bool same = g + 1 < TPL / GRP;
            const int jn0 = same ? j0 : j0 + EXM_DCH;
            const int gn = same ? (g + 1) * GRP : 0;
            if (same || j0 + EXM_DCH < end) {
#pragma unroll
                for (int u = 0; u < GRP; ++u) {
                    const int jl = jn0 + TPL * lane + gn + u;
                    qa[u] = (jl >= beg && jl < end) ? __ldg(c.descr + jn0 + 32 * (gn + u) + lane)
                                                    : make_uint4(0u, 0u, 0u, 0u);
                }
            }
            tap_group<BND, GRP, TE>(a, c, cur, jb + g * GRP, j0 + 32 * g * GRP + lane, beg, end, cT, cB, cE, cS, fT,
                                    fB, fE, fS, n_slow);
        }
        // the first closed template of lane l + 1 continues lane l's last one, or is lane l + 1's alone
        const int nT = __shfl_down_sync(0xffffffffu, fT, 1);
        const float nB = __shfl_down_sync(0xffffffffu, fB, 1);
        const float nE = __shfl_down_sync(0xffffffffu, fE, 1);
        const float nS = __shfl_down_sync(0xffffffffu, fS, 1);
        const int pT = __shfl_up_sync(0xffffffffu, cT, 1);
        if (lane < 31 && nT >= 0 && nT == cT) lse_merge(cB, cE, cS, nB, nE, nS);
        if (fT >= 0 && !(lane > 0 && pT == fT)) acc_merge(c, fT, fB, fE, fS);
        // last templates: runs across consecutive lanes
        const bool head = seg_reduce(cT >= 0 ? cT : -2 - lane, cB, cE, cS);
        if (head && cT >= 0) acc_merge(c, cT, cB, cE, cS);
    }
}

// the template of the descriptor at sorted position j (block-local), or -1
__device__ __forceinline__ int desc_template(const RunCtx &c, int j)
{
    return (int)(__ldg(&c.descr[exm_desc_phys(j)].w) >> 19) + c.m_base - c.lo;
}

// fold the warps' edge partials into the accumulators: one warp, lane w holding warp w's first (F)
// and last (L) partials; templates ascend along the warps, so this is the lane-level merge again
__device__ __forceinline__ void fold_edges(float *edge, int nw, float *aB, float *aE, float *aS, int n)
{
    const int lane = threadIdx.x & 31;
    float fB = -1e30f, fE = 0.f, fS = 0.f, cB = -1e30f, cE = 0.f, cS = 0.f;
    int fT = -1, cT = -1;
    if (lane < nw) {
        const float *e = edge + 8 * lane;
        fT = __float_as_int(e[3]);
        fB = e[0];
        fE = e[1];
        fS = e[2];
        cT = __float_as_int(e[7]);
        cB = e[4];
        cE = e[5];
        cS = e[6];
        if (!(fT >= 0 && fT < n && fS > 0.f)) fT = -1;
        if (!(cT >= 0 && cT < n)) cT = -1;
    }
    const int nT = __shfl_down_sync(0xffffffffu, fT, 1);
    const float nB = __shfl_down_sync(0xffffffffu, fB, 1);
    const float nE = __shfl_down_sync(0xffffffffu, fE, 1);
    const float nS = __shfl_down_sync(0xffffffffu, fS, 1);
    const int pT = __shfl_up_sync(0xffffffffu, cT, 1);
    if (lane < 31 && nT >= 0 && nT == cT) lse_merge(cB, cE, cS, nB, nE, nS);
    if (fT >= 0 && !(lane > 0 && pT == fT)) {
        float b = aB[fT], x = aE[fT], q = aS[fT];
        lse_merge(b, x, q, fB, fE, fS);
        aB[fT] = b;
        aE[fT] = x;
        aS[fT] = q;
    }
    const bool head = seg_reduce(cT >= 0 ? cT : -2 - lane, cB, cE, cS);
    if (head && cT >= 0 && cS > 0.f) {
        float b = aB[cT], x = aE[cT], q = aS[cT];
        lse_merge(b, x, q, cB, cE, cS);
        aB[cT] = b;
        aE[cT] = x;
        aS[cT] = q;
    }
}

// this warp's equal share [w0, w1) of the run [beg, end), with its edge templates and slots
template <bool BND, int GRP, int NW, typename TE>
__device__ __forceinline__ void warp_share(const PlaneArgs &a, RunCtx &c, int beg, int end, unsigned edge, int pair,
                                           unsigned &n_slow)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // whole storage chunks per warp, as evenly as they divide (the first and last may be partial).
    // The warps with work are a prefix: the edge fold merges equal templates of neighbouring lanes
    // only, so an empty warp between two that share a template would let both update its
    // accumulator at once.  When every warp has a chunk, the rem warps that take one more are a
    // cyclic window that moves by rem with the pair, so that no warp takes the extra chunk at every
    // pair: a warp runs at most one pair ahead, so with a fixed prefix the others would wait at every pair.
    const int cb = beg / EXM_DCH, nc = (end + EXM_DCH - 1) / EXM_DCH - cb;
    const int q = nc / NW, rem = nc % NW;
    const int s = q > 0 ? (pair * rem) % NW : 0, se = s + rem;
    const int before = max(0, min(warp, se) - s) + max(0, min(warp, se - NW));   // extra chunks of warps < warp
    const int c0 = cb + warp * q + before, c1 = c0 + q + ((warp - s + NW) % NW < rem ? 1 : 0);
    const int w0 = max(beg, c0 * EXM_DCH), w1 = min(end, c1 * EXM_DCH);
    const unsigned eo = edge + 32u * warp;   // 8 floats per warp
    float *e = gsm_f(eo);
    int tF = -1, tL = -1;
    if (w0 < w1) {
        tF = desc_template(c, w0);
        tL = desc_template(c, w1 - 1);
    }
    if (lane == 0) {
        e[0] = -1e30f;
        e[1] = 0.f;
        e[2] = 0.f;
        e[3] = __int_as_float(tF == tL ? -1 : tF);
        e[4] = -1e30f;
        e[5] = 0.f;
        e[6] = 0.f;
        e[7] = __int_as_float(tL);
    }
    __syncwarp();
    c.tF = (tF == tL) ? -1 : tF;   // one template only: the L slot takes it all
    c.tL = tL;
    c.eF = eo;
    c.eL = eo + 16u;
    if (w0 < w1) process_run<BND, GRP, TE>(a, c, w0, w1, n_slow);
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Warp NW - 1 is the producer: it stages the planes with TMA and, once every consumer warp has
// arrived on the pair's "done" barrier, folds that pair's edge partials and refills the slot of
// the plane no longer needed.  The NW - 1 consumer warps walk the pairs without a block barrier:
// a fast warp runs at most one pair ahead of the slowest (pair p + 2 needs plane p + 3, staged
// only after pair p is done everywhere).  So at most two consecutive pairs are in flight, and the
// consumers' accumulators alternate with the pair's parity (two warps in different pairs never
// share a word), while the producer folds edges into a third set of its own.
template <int NW, int GRP, typename TE>
__global__ void __launch_bounds__(NW * 32, 1) k_gather_planes(const __grid_constant__ CUtensorMap tmap,
                                                                const __grid_constant__ PlaneArgs a)
{
    constexpr int NC = NW - 1;   // consumer warps
    constexpr int SLOT = slot_elems<TE>();
    constexpr unsigned SLOT_B = slot_bytes<TE>();
    unsigned char *smem = exm_gsm;
    TE *win = (TE *)smem;
    uint64_t *full = (uint64_t *)(smem + 3 * SLOT_B);   // [3] plane staged in slot s
    uint64_t *done = full + 3;                          // [2] every consumer is done with a pair (parity)
    const int tch = a.tch;
    // accumulator sets of 3 x tch floats (B, E, S): regular pairs of parity 0 / 1, regular edges
    // (producer), boundary pairs of parity 0 / 1, boundary edges; then bcf, bsh; then the edge
    // slots [pair parity][regular, boundary][8 floats per consumer warp: F and L partials + ids]
    const unsigned acc_o = 3 * SLOT_B + 64;
    float *acc = gsm_f(acc_o);
    float *bcf = acc + 18 * tch;
    int *bsh = (int *)(bcf + tch);
    const unsigned bcf_o = acc_o + 4u * 18u * tch, bsh_o = bcf_o + 4u * tch, edge_o = bsh_o + 4u * tch;
    // exact-path queues [pair mod 3][consumer warp]: counts, then EXM_SLOWQ int2 entries (storage index of the
    // tap; template | boundary flag << 30 | random-draw flag << 29)
    const unsigned qcnt_o = edge_o + 4u * (2 * 2 * 8 * 32), qent_o = qcnt_o + 4u * 3 * 32;
    int *qcnt = (int *)(smem + qcnt_o);
    const int2 *qent = (const int2 *)(smem + qent_o);
    auto edge_off = [&](int par, int b2) { return edge_o + 4u * (unsigned)((par * 2 + b2) * 8 * NC); };
    __shared__ int bl_sh[2];
    __shared__ unsigned bad_sh;

    // block -> (lag, node, template chunk), lags outermost so the blocks of one lag run together
    const int c_idx = blockIdx.x % a.nch;
    const int k = (blockIdx.x / a.nch) % a.nn;
    const int rl = blockIdx.x / (a.nch * a.nn), r = a.r0 + rl;
    const int lo0 = max(a.mlo[k], a.m_base), hi0 = min(a.mhi[k], a.m_base + a.nmc);
    const int lo = lo0 + c_idx * tch;
    const int hi = min(hi0, lo + tch);
    if (lo >= hi) return;
    const int n = hi - lo;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    if (tid == 0) {
        bl_sh[0] = n;
        bl_sh[1] = 0;
        bad_sh = 0;
    }
    __syncthreads();
    // the node's window: column C0, first row R0 = Rh + cki clamped to the table; a tap's window row
    // is its beta-hat row from Rh (in the descriptor), plus the carry of the node's beta fraction, plus sh
    const int C0 = a.win[0], R0 = a.win[1 + k], Rh = a.win[1 + EXM_MAX_NODES];
    const int sh = Rh + a.cki[k] - R0;
    for (int j = tid; j < n; j += NW * 32) {
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            acc[(3 * q) * tch + j] = -1e30f;
            acc[(3 * q + 1) * tch + j] = 0.f;
            acc[(3 * q + 2) * tch + j] = 0.f;
        }
        bsh[j] = EXM_BSH_NONE;
        if (a.bnode[lo + j] == k) {
            const double cbv = a.cb[lo + j];
            const double f = floor(cbv);
            bsh[j] = (int)f - a.cki[k] + sh;
            bcf[j] = (float)(cbv - f);
            atomicMin(&bl_sh[0], j);
            atomicMax(&bl_sh[1], j + 1);
        }
    }
    if (tid == 0) {
        for (int s = 0; s < 3; ++s) mbar_init(&full[s], 1);
        for (int s = 0; s < 2; ++s) mbar_init(&done[s], NC * 32);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const int blo = bl_sh[0], bhi = bl_sh[1];
    unsigned n_slow = 0, n_bnd = 0;

    if (warp == NC) {
        // ---------------------------------------------------------------- producer
        const int32_t *tsr_all = a.tside + (long long)rl * a.per_lag;
        int issued = 0;
        if (a.stage) {
            if (lane == 0)
                for (int q = 0; q < 3 && q < a.nphif; ++q)
                    tma_load_plane(&tmap, &full[q], win + q * SLOT, C0, R0, q, r, k, SLOT_B);
            issued = min(3, a.nphif);
        }
        bool ok = true;
        for (int p = 0; p < EXM_NPAIR; ++p) {
            ok = ok && __all_sync(0xffffffffu, mbar_wait(&done[p & 1], (p >> 1) & 1, a.err, a.wait_cycles));
            if (!ok) break;
            fold_edges(gsm_f(edge_off(p & 1, 0)), NC, acc + 6 * tch, acc + 7 * tch, acc + 8 * tch, n);
            if (blo < bhi)
                fold_edges(gsm_f(edge_off(p & 1, 1)), NC, acc + 15 * tch, acc + 16 * tch, acc + 17 * tch, n);
            __syncwarp();
            // plane p is no longer needed anywhere: its slot takes plane p + 3
            if (a.stage && p + 3 < a.nphif) {
                if (lane == 0) tma_load_plane(&tmap, &full[p % 3], win + (p % 3) * SLOT, C0, R0, p + 3, r, k, SLOT_B);
                ++issued;
            }
            // the exact-path taps the consumers queued for pair p: 32 lanes compute them, lane 0 merges them
            // in warp and queue order into the producer's sets (the consumers reuse these queues at pair
            // p + 3, after plane p + 4, which is staged only after this)
            {
                const int par = p % 3;
                const int cw = lane < NC ? qcnt[par * 32 + lane] : 0;
                int incl = cw;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += y;
                }
                const int total = __shfl_sync(0xffffffffu, incl, 31);
                const int excl = incl - cw;
                for (int b0 = 0; b0 < total; b0 += 32) {
                    const int i = b0 + lane;
                    double v = 0.0;
                    int tr = 0, bnd = 0;
                    int wi = 0;   // the warp whose entries [excl, incl) hold i (shuffles kept converged)
                    for (int l = 1; l < NC; ++l) {
                        const int el = __shfl_sync(0xffffffffu, excl, l);
                        wi += (i < total && el <= i) ? 1 : 0;
                    }
                    const int wexcl = __shfl_sync(0xffffffffu, excl, wi);
                    if (i < total) {
                        const int2 e = qent[(par * 32 + wi) * EXM_SLOWQ + (i - wexcl)];
                        const int il = e.y & 0x1FFF;
                        bnd = (e.y >> 30) & 1;
                        const int tm = tsr_all[e.x];
                        v = bnd ? slow_tap<true, TE>(a, il, tm, k, r, a.m_base, a.tsc[k])
                                : slow_tap<false, TE>(a, il, tm, k, r, a.m_base, a.tsc[k]);
                        v += ((e.y >> 29) & 1) ? (double)a.lw : 0.0;
                        tr = il + a.m_base - lo;
                    }
                    const int nb2 = min(32, total - b0);
                    for (int qq = 0; qq < nb2; ++qq) {
                        const double vq = __shfl_sync(0xffffffffu, v, qq);
                        const int tq = __shfl_sync(0xffffffffu, tr, qq), bq = __shfl_sync(0xffffffffu, bnd, qq);
                        if (lane == 0 && tq >= 0 && tq < n) {
                            float B, E;
                            split_double(vq, B, E);
                            float *F = acc + (bq ? 15 : 6) * tch;
                            float b = F[tq], x = F[tch + tq], sv = F[2 * tch + tq];
                            lse_merge(b, x, sv, B, E, 1.f);
                            F[tq] = b;
                            F[tch + tq] = x;
                            F[2 * tch + tq] = sv;
                        }
                    }
                }
                __syncwarp();
            }
        }
        if (!ok) {
            if (lane == 0) {
                atomicOr(&bad_sh, 1u);
                // drain: the newest copy of each slot completes after the older ones of that slot (bounded by
                // the full limit whatever the pipeline's: the block must not exit with a copy in flight)
                for (int q = max(0, issued - 3); q < issued; ++q) mbar_wait(&full[q % 3], (q / 3) & 1, a.err);
            }
        }
    } else {
        // ---------------------------------------------------------------- consumers
        const int *offr = a.off + (long long)rl * EXM_NPAIR * (a.nmc + 1);
        RunCtx rc;
        rc.descr = a.desc + (long long)rl * a.per_lag;
        rc.tsr = a.tside + (long long)rl * a.per_lag;
        rc.bsh = bsh_o;
        rc.bcf = bcf_o;
        rc.accst = 4u * tch;
        rc.lo = lo;
        rc.m_base = a.m_base;
        rc.n = n;
        rc.sh = sh;
        rc.up = min(EXM_WB - 2, a.nb - 2 - R0);
        rc.edge = a.nb - 2 - R0;
        rc.ckf = a.ckf[k];
        rc.sc = a.tsc[k];
        rc.k = k;
        rc.r = r;
        rc.lw = a.lw;
        const int base_i = lo - a.m_base;   // chunk-local index of template lo
        bool ok = true;
        for (int p = 0; p < EXM_NPAIR; ++p) {
            // warp-uniform: the lanes go on to shuffles together
            ok = ok && __all_sync(0xffffffffu, mbar_wait(&full[p % 3], (p / 3) & 1, a.err, a.wait_cycles));
            ok = ok && __all_sync(0xffffffffu,
                                  mbar_wait(&full[(p + 1) % 3], ((p + 1) / 3) & 1, a.err, a.wait_cycles));
            if (lane == 0) qcnt[(p % 3) * 32 + warp] = 0;
            __syncwarp();
            rc.qn = qcnt_o + 4u * ((p % 3) * 32 + warp);
            rc.q = qent_o + 8u * (((p % 3) * 32 + warp) * EXM_SLOWQ);
            if (ok) {
                rc.s0 = (p % 3) * SLOT_B;
                rc.s1 = ((p + 1) % 3) * SLOT_B;
                const int *offp = offr + p * (a.nmc + 1) + base_i;
                rc.acc = acc_o + 4u * (3u * (p & 1) * tch);
                warp_share<false, GRP, NC, TE>(a, rc, offp[0], offp[n], edge_off(p & 1, 0), p, n_slow);
                if (blo < bhi) {
                    rc.acc = acc_o + 4u * ((9u + 3u * (p & 1)) * tch);
                    const int bb = offp[blo], be = offp[bhi];
                    n_bnd += (lane == 0 && warp == 0) ? (unsigned)(be - bb) : 0u;
                    warp_share<true, GRP, NC, TE>(a, rc, bb, be, edge_off(p & 1, 1), p, n_slow);
                }
            } else if (lane == 0) {   // no work: empty edge slots for the producer
                for (int b2 = 0; b2 < 2; ++b2) {
                    float *e = gsm_f(edge_off(p & 1, b2)) + 8 * warp;
                    e[3] = __int_as_float(-1);
                    e[7] = __int_as_float(-1);
                }
            }
            __syncwarp();
            mbar_arrive(&done[p & 1]);
        }
        if (!ok && lane == 0) atomicOr(&bad_sh, 1u);
    }
    if (a.stats) {
        const unsigned sl_ = __reduce_add_sync(0xffffffffu, n_slow), bd_ = __reduce_add_sync(0xffffffffu, n_bnd);
        if (lane == 0 && (sl_ | bd_)) {
            atomicAdd(&a.stats[0], (unsigned long long)sl_);
            atomicAdd(&a.stats[1], (unsigned long long)bd_);
        }
    }
    __syncthreads();
    const bool ok = bad_sh == 0;
    for (int j = tid; j < n; j += NW * 32) {
        // the three sets of a template: both pair parities and the folded edges
        float B = acc[j], E = acc[tch + j], S = acc[2 * tch + j];
        lse_merge(B, E, S, acc[3 * tch + j], acc[4 * tch + j], acc[5 * tch + j]);
        lse_merge(B, E, S, acc[6 * tch + j], acc[7 * tch + j], acc[8 * tch + j]);
        const double v = (ok && S > 0.f) ? (double)B + (double)E + log((double)S) : -INFINITY;
        a.part[((long long)k * a.ntau + r) * a.nm_total + lo + j] = v;
        if (j >= blo && j < bhi && a.bnode[lo + j] == k) {
            float B2 = acc[9 * tch + j], E2 = acc[10 * tch + j], S2 = acc[11 * tch + j];
            lse_merge(B2, E2, S2, acc[12 * tch + j], acc[13 * tch + j], acc[14 * tch + j]);
            lse_merge(B2, E2, S2, acc[15 * tch + j], acc[16 * tch + j], acc[17 * tch + j]);
            const double v2 = (ok && S2 > 0.f) ? (double)B2 + (double)E2 + log((double)S2) : -INFINITY;
            a.part[((long long)a.nn * a.ntau + r) * a.nm_total + lo + j] = v2;
        }
    }
}

// launch shapes the autotuner chooses from: (warps per block, taps per register group)
struct GatherCfg {
    int nw, grp;
};
// warps incl. producer x taps per register group; the first is the default of an untuned context
static const GatherCfg kGatherCfgs[] = {{28, 1}, {16, 2}, {24, 2}, {24, 1}, {20, 2}};
static const int kNumGatherCfgs = (int)(sizeof(kGatherCfgs) / sizeof(kGatherCfgs[0]));

template <int NW, int GRP0, typename TE>
static void launch_planes(exm_ctx *ctx, const PlaneArgs &a, dim3 grid, size_t smem)
{
    constexpr int GRP = GRP0 < TPL ? GRP0 : TPL;   // a register group never exceeds a lane's taps
    exm_allow_smem(ctx, (const void *)k_gather_planes<NW, GRP, TE>, smem);
    k_gather_planes<NW, GRP, TE><<<grid, NW * 32, smem, ctx->stream>>>(ctx->tmap, a);
}

template <typename TE>
static void launch_cfg_t(exm_ctx *ctx, int cfg, const PlaneArgs &a, dim3 grid, size_t smem)
{
    switch (cfg) {
    case 0: launch_planes<28, 1, TE>(ctx, a, grid, smem); break;
    case 1: launch_planes<16, 2, TE>(ctx, a, grid, smem); break;
    case 2: launch_planes<24, 2, TE>(ctx, a, grid, smem); break;
    case 3: launch_planes<24, 1, TE>(ctx, a, grid, smem); break;
    default: launch_planes<20, 2, TE>(ctx, a, grid, smem); break;
    }
}

static void launch_cfg(exm_ctx *ctx, int cfg, const PlaneArgs &a, dim3 grid, size_t smem)
{
    if (ctx->dtype == EXM_DTYPE_F16)
        launch_cfg_t<__half>(ctx, cfg, a, grid, smem);
    else if (ctx->dtype == EXM_DTYPE_BF16)
        launch_cfg_t<__nv_bfloat16>(ctx, cfg, a, grid, smem);
    else
        launch_cfg_t<float>(ctx, cfg, a, grid, smem);
}

int exm_gather_num_cfgs() { return kNumGatherCfgs; }

static size_t planes_smem(int tch, int dtype)
{
    const size_t slot = (size_t)EXM_WB * exm_dtype_wd(dtype) * exm_dtype_bytes(dtype);
    // 6 accumulator sets of 3 floats, bcf, bsh; edge slots; exact-path queue counts and entries
    return 3 * slot + 64 + (size_t)tch * 20 * 4 + 2 * 2 * 8 * 32 * 4 + 3 * 32 * 4 + 3 * 32 * EXM_SLOWQ * 8;
}

// the most templates a block can hold in shared memory next to the staged planes
static int planes_tch_max(exm_ctx *ctx)
{
    const size_t slot = (size_t)EXM_WB * exm_dtype_wd(ctx->dtype) * exm_dtype_bytes(ctx->dtype);
    const size_t fixed = 3 * slot + 64 + 2 * 2 * 8 * 32 * 4 + 3 * 32 * 4 + 3 * 32 * EXM_SLOWQ * 8 + 2048;   // + static
    const size_t room = ctx->smem_optin > fixed ? ctx->smem_optin - fixed : 0;
    return (int)std::min<size_t>(EXM_TCH, room / (20 * 4) / 16 * 16);
}

void exm_run_gather_planes(exm_ctx *ctx, exm_slot &sl, const ChunkInfo &ci, int r0, int rc)
{
    if (!ctx->tmap_ok) EXM_THROW(EXM_ERR_STATE, "tensor map of the store is not set");
    PlaneArgs a;
    memset(&a, 0, sizeof(a));
    a.desc = (const uint4 *)sl.desc.p;
    a.tside = (const int32_t *)sl.tside.p;
    a.off = (const int *)sl.cnt.p;
    a.H = (const float2 *)sl.traj.p;
    a.L = a.H + (size_t)ci.nmc * ctx->nt;
    a.Hlo = ctx->traj_fp64 ? (const float *)sl.trajlo.p : nullptr;
    a.Llo = a.Hlo ? a.Hlo + (size_t)ci.nmc * ctx->nt : nullptr;
    a.T = ctx->T.p;
    a.mlo = (const int *)ctx->d_mlo.p;
    a.mhi = (const int *)ctx->d_mhi.p;
    a.bnode = (const int *)ctx->d_bnode.p;
    a.win = (const int *)sl.win.p;
    a.tau = (const int *)ctx->d_tau.p;
    a.boff = (const double *)ctx->d_bhat_off.p;
    a.cb = (const double *)ctx->d_cb.p;
    a.ckd = (const double *)ctx->d_ckd.p;
    a.part = (double *)sl.part.p;
    a.err = (unsigned *)sl.dev_err.p;
    a.stats = (unsigned long long *)ctx->d_stats.p;
    a.tstride = (long long)ctx->tstride;
    a.per_lag = exm_desc_pitch((long long)ci.nmc * ci.nwalk);   // storage stride of a lag's descriptors
    a.nn = ctx->nn;
    a.ntau = ctx->ntau;
    a.nphif = ctx->nphif;
    a.nb = ctx->nb;
    a.nd = ctx->nd;
    a.ndp = ctx->ndp;
    a.nt = ctx->nt;
    a.nmc = ci.nmc;
    a.m_base = ci.m_base;
    a.nm_total = ctx->nm;
    a.r0 = r0;
    a.lw = ci.lw;
    a.rph = EXM_NPHI / 6.283185307179586;
    a.rdb = 2.0 / ctx->dbeta;
    a.rdd = 1.0 / ctx->ddelta;
    a.offd = -ctx->delta0 / ctx->ddelta;
    a.stage = ctx->test_wait_expiry ? 0 : 1;
    a.wait_cycles = ctx->test_wait_expiry ? EXM_TEST_WAIT_CYCLES : EXM_WAIT_CYCLES;
    for (int k = 0; k < ctx->nn; ++k) {
        const double f = std::floor(ctx->ck[k]);
        a.cki[k] = (int)f;
        a.ckf[k] = (float)(ctx->ck[k] - f);
        a.tsc[k] = ctx->tscale[k];
    }
    // templates per block: about one wave of blocks per lag, so that the descriptors of the lag
    // in flight stay in L2; at most EXM_TCH (shared-memory accumulators)
    long long pairs = 0;
    int maxn = 0;
    for (int k = 0; k < ctx->nn; ++k) {
        const int lo = std::max(ctx->mlo[k], ci.m_base), hi = std::min(ctx->mhi[k], ci.m_base + ci.nmc);
        pairs += std::max(0, hi - lo);
        maxn = std::max(maxn, hi - lo);
    }
    if (maxn <= 0) return;
    int tch = (int)((pairs + ctx->sm_count - 1) / ctx->sm_count);
    tch = (int)((long long)tch * ctx->gather_chunk_pct / 100);
    tch = std::max(tch, 256);
    tch = std::min(((tch + 15) / 16) * 16, planes_tch_max(ctx));
    a.tch = tch;
    a.nch = (maxn + tch - 1) / tch;
    const size_t smem = planes_smem(tch, ctx->dtype);
    dim3 grid(rc * ctx->nn * a.nch);
    const int cfg = (ctx->gather_cfg >= 0 && ctx->gather_cfg < kNumGatherCfgs) ? ctx->gather_cfg : 0;
    launch_cfg(ctx, cfg, a, grid, smem);
    EXM_CUDA(cudaGetLastError());
    // algorithmic work of this launch: one node-tap per (template slot, lag, walked time)
    double slots = 0;
    for (int k = 0; k < ctx->nn; ++k) {
        const int lo = std::max(ctx->mlo[k], ci.m_base), hi = std::min(ctx->mhi[k], ci.m_base + ci.nmc);
        slots += std::max(0, hi - lo);
    }
    for (int i = ci.m_base; i < ci.m_base + ci.nmc; ++i) slots += ctx->bnode[i] >= 0;
    ctx->node_taps += slots * rc * ci.nwalk;
    ctx->tlw += (double)ci.nmc * rc * ci.nwalk;
    ctx->gather_launches += 1;
    ctx->launches += 1;
}

// ------------------------------------------------------------------ the general gather contract, float64

struct SimpleArgs {
    const float2 *H, *L;
    const float *Hlo, *Llo;
    const int32_t *sel;
    const void *T;              // node tables (element type TE of the kernel)
    const float *tsc;           // per node scale
    const int *rows, *tab, *tau;
    const double *lna;
    double *om, *os;
    long long tstride;
    int nt, nwalk, use_sel, ns, nsel, nphif, nb, nd, ndp, ntau;
    float lw;
    double beta0, dbeta, rph, rdb, rdd, offd;
};

template <typename TE>
__global__ void __launch_bounds__(256) k_gather_simple(SimpleArgs a)
{
    __shared__ double shm[8], shs[8];
    const int j = blockIdx.x, r = blockIdx.y;
    const int row = a.rows[j];
    const int nt = a.nt;
    const int tau0 = ((a.tau[r] % nt) + nt) % nt;
    const float2 *H = a.H + (long long)row * nt, *L = a.L + (long long)row * nt;
    const float *Hlo = a.Hlo ? a.Hlo + (long long)row * nt : nullptr, *Llo = a.Llo ? a.Llo + (long long)row * nt : nullptr;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int n = 0; n < a.ns; ++n) {
        const int tb = a.tab[j * a.ns + n];
        const TE *Tn = (const TE *)a.T + (long long)tb * a.tstride;
        const float sc = a.tsc[tb];
        const double offb = (a.lna[j * a.ns + n] - a.beta0) / a.dbeta;
        double m = -1e300, s = 0.0;
        for (int kk = threadIdx.x; kk < a.nwalk; kk += blockDim.x) {
            int t = kk, flag = 0;
            if (a.use_sel) {
                const int v = a.sel[(long long)row * a.nwalk + kk];
                t = v & 0x7FFFFFFF;
                flag = (unsigned)v >> 31;
            }
            int i1 = t + tau0;
            if (i1 >= nt) i1 -= nt;
            double acc = exm_tap_fp64<TE>(L[t], H[i1], Llo ? Llo[t] : 0.f, Hlo ? Hlo[i1] : 0.f, offb, r, Tn, sc, a.nphif, a.nb, a.nd, a.ndp, a.rph, a.rdb,
                                          a.rdd, a.offd);
            if (a.use_sel) acc += flag ? (double)a.lw : 0.0;
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

__global__ void k_lse_lags(const double *om, const double *os, int ns, int ntau, int nsel, int nt, double *out)
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

void exm_run_gather_simple(exm_ctx *ctx, exm_slot &sl, int nsel, int ns, const int *d_rows, const int *d_tab,
                           const double *d_lna, int nwalk, int use_sel, float lw, double *d_out)
{
    SimpleArgs a;
    a.H = (const float2 *)sl.traj.p;
    a.L = a.H + (size_t)ctx->nm * ctx->nt;
    a.Hlo = ctx->traj_fp64 ? (const float *)sl.trajlo.p : nullptr;
    a.Llo = a.Hlo ? a.Hlo + (size_t)ctx->nm * ctx->nt : nullptr;
    a.sel = (const int32_t *)sl.sel.p;
    a.T = ctx->T.p;
    a.tsc = (const float *)ctx->d_tscale.p;
    a.rows = d_rows;
    a.tab = d_tab;
    a.tau = (const int *)ctx->d_tau.p;
    a.lna = d_lna;
    a.om = (double *)sl.part.p;
    a.os = a.om + (size_t)ns * ctx->ntau * nsel;
    a.tstride = (long long)ctx->tstride;
    a.nt = ctx->nt;
    a.nwalk = nwalk;
    a.use_sel = use_sel;
    a.ns = ns;
    a.nsel = nsel;
    a.nphif = ctx->nphif;
    a.nb = ctx->nb;
    a.nd = ctx->nd;
    a.ndp = ctx->ndp;
    a.ntau = ctx->ntau;
    a.lw = lw;
    a.beta0 = ctx->beta0;
    a.dbeta = ctx->dbeta;
    a.rph = EXM_NPHI / 6.283185307179586;
    a.rdb = 2.0 / ctx->dbeta;
    a.rdd = 1.0 / ctx->ddelta;
    a.offd = -ctx->delta0 / ctx->ddelta;
    dim3 grid(nsel, ctx->ntau);
    if (ctx->dtype == EXM_DTYPE_F16)
        k_gather_simple<__half><<<grid, 256, 0, ctx->stream>>>(a);
    else if (ctx->dtype == EXM_DTYPE_BF16)
        k_gather_simple<__nv_bfloat16><<<grid, 256, 0, ctx->stream>>>(a);
    else
        k_gather_simple<float><<<grid, 256, 0, ctx->stream>>>(a);
    k_lse_lags<<<(ns * nsel + 255) / 256, 256, 0, ctx->stream>>>(a.om, a.os, ns, ctx->ntau, nsel, ctx->nt, d_out);
    EXM_CUDA(cudaGetLastError());
}
