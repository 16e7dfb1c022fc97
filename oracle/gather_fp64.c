/*
 * ORACLE -- test infrastructure only.  Tests, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py call this as the checker; the
 * product never links or calls it.
 *
 * Plain-C restatement of the reference's CPU table read, Eq. (C7):
 *   exmarg/search/gather.py:32-100  (_gather_cpu, the per (template, lag) job)
 *   exmarg/search/gather.py:103-107 (_lse_lags, the log-sum-exp over lags)
 *   exmarg/search/gather.py:110-111 (_offsets)
 * Every intermediate is float64, the table values are the stored float32.
 * The (template, lag) jobs run in parallel over the host cores (OpenMP), as
 * the reference's numba prange does.
 *
 * Build: gcc -O2 -fopenmp -shared -fPIC (oracle/build_oracle.py).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define NPHI 96

/*
 * lq*, ph*   (n_template, n_time) float64: ln|z| and arg z of H and L
 * mass_ids   (nsel,) template rows
 * tab_ids    (nsel, ns) index into tables[] of each (template, slot)
 * lna        (nsel, ns) ln a of each (template, slot)
 * tau_idx    (ntau,) lags in samples
 * tables     ntab pointers to float32 (ntau, nphif, nb, nd) C-order tables
 * sel, lw    (n_template, nwalk) visited times and log weights, or NULL (all times)
 * phase_f32  1: the phase difference in float32, as the reference (float32 trajectories)
 * out        (ns, nsel) float64: ln Lambda = LSE over lags of the running (max, sum) - ln n_time
 */
int oracle_gather(int n_time, const double *lqH, const double *phH, const double *lqL, const double *phL,
                  int nsel, int ns, const int64_t *mass_ids, const int64_t *tab_ids, const double *lna,
                  int ntau, const int64_t *tau_idx, const float *const *tables, int nphif, int nb, int nd,
                  double beta0, double dbeta, double delta0, double ddelta,
                  int nwalk, const int32_t *sel, const float *lw, int phase_f32, double *out)
{
    const double rph = NPHI / 6.283185307179586;
    const double rdb = 2.0 / dbeta;
    const double offd = -delta0 / ddelta;
    const double rdd = 1.0 / ddelta;
    const int use_sel = (sel != NULL);
    const int nw = use_sel ? nwalk : n_time;
    double *om = (double *)malloc(sizeof(double) * (size_t)ns * ntau * nsel);
    double *os = (double *)malloc(sizeof(double) * (size_t)ns * ntau * nsel);
    if (!om || !os) { free(om); free(os); return 1; }
    const int64_t njob = (int64_t)nsel * ntau;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t job = 0; job < njob; ++job) {
        const int j = (int)(job / ntau), r = (int)(job % ntau);
        const int64_t mid = mass_ids[j];
        const int64_t tau0 = ((tau_idx[r] % n_time) + n_time) % n_time;
        const double *lH = lqH + mid * n_time, *pH = phH + mid * n_time;
        const double *lL = lqL + mid * n_time, *pL = phL + mid * n_time;
        for (int n = 0; n < ns; ++n) {
            const float *Tn = tables[tab_ids[(int64_t)j * ns + n]];
            const double offb = (lna[(int64_t)j * ns + n] - beta0) / dbeta;
            double m = -1e300, s = 0.0;
            for (int k = 0; k < nw; ++k) {
                const int64_t t = use_sel ? sel[mid * nwalk + k] : k;
                int64_t i1 = t + tau0;
                if (i1 >= n_time) i1 -= n_time;
                /* the reference subtracts the two float32 phases in float32 (numba keeps the
                   array type), then scales in float64; phase_f32 = 0 keeps everything float64 */
                double x3 = phase_f32 ? (double)((float)pH[i1] - (float)pL[t]) * rph : (pH[i1] - pL[t]) * rph;
                if (x3 < 0.0) x3 += NPHI;
                if (x3 >= NPHI) x3 -= NPHI;
                int c0 = (int)x3;
                if (c0 >= NPHI) c0 = NPHI - 1; else if (c0 < 0) c0 = 0;
                const double fc = x3 - c0;
                const int c1 = (c0 + 1) % NPHI;
                const double aH = lH[i1], aL = lL[t];
                const double xbr = aL * rdb + offb;
                double xb = xbr;
                if (xb < 0.0) xb = 0.0; else if (xb > nb - 1 - 1e-6) xb = nb - 1 - 1e-6;
                const double aLc = aL + (xb - xbr) / rdb;
                double xd = (aH - aLc) * rdd + offd;
                if (xd < 0.0) xd = 0.0; else if (xd > nd - 1 - 1e-6) xd = nd - 1 - 1e-6;
                const int d0 = (int)xd; const double fdf = xd - d0, fd0 = 1.0 - fdf;
                const int d1 = d0 + 1 < nd ? d0 + 1 : nd - 1;
                const int b0 = (int)xb; const double fbf = xb - b0, fb0 = 1.0 - fbf;
                const int b1 = b0 + 1 < nb ? b0 + 1 : nb - 1;
                double acc = 0.0;
                for (int cc = 0; cc < 2; ++cc) {
                    int ci = cc ? c1 : c0;
                    if (ci > NPHI / 2) ci = NPHI - ci;
                    const double fci = cc ? fc : 1.0 - fc;
                    const float *row0 = Tn + (((int64_t)r * nphif + ci) * nb + b0) * nd;
                    const float *row1 = Tn + (((int64_t)r * nphif + ci) * nb + b1) * nd;
                    const double v = fb0 * (fd0 * row0[d0] + fdf * row0[d1]) + fbf * (fd0 * row1[d0] + fdf * row1[d1]);
                    acc += fci * v;
                }
                if (use_sel) acc += (double)lw[mid * nwalk + k];
                if (acc > m) { s = s * exp(m - acc) + 1.0; m = acc; }
                else s += exp(acc - m);
            }
            om[((int64_t)n * ntau + r) * nsel + j] = m;
            os[((int64_t)n * ntau + r) * nsel + j] = s;
        }
    }
    const double lnt = log((double)n_time);
    for (int n = 0; n < ns; ++n)
        for (int j = 0; j < nsel; ++j) {
            double mx = -INFINITY;
            for (int r = 0; r < ntau; ++r) {
                const double v = om[((int64_t)n * ntau + r) * nsel + j];
                if (v > mx) mx = v;
            }
            double tot = 0.0;
            for (int r = 0; r < ntau; ++r) {
                const int64_t o = ((int64_t)n * ntau + r) * nsel + j;
                tot += os[o] * exp(om[o] - mx);
            }
            out[(int64_t)n * nsel + j] = mx + log(tot) - lnt;
        }
    free(om);
    free(os);
    return 0;
}

int oracle_num_threads(void)
{
    int n = 1;
#pragma omp parallel
    {
#pragma omp single
        {
#ifdef _OPENMP
            n = omp_get_num_threads();
#endif
        }
    }
    return n;
}
