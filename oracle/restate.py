"""ORACLE -- test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs
import this module, and only as the checker (or as the timed CPU baseline).  The
exmarg_b200 package never imports it.

A restatement, in plain numpy plus the C gather of gather_fp64.c, of the
reference's pe_intrinsic path.  Each function cites the reference code it follows.
Two precisions:

* precision='fp64': every step in float64 (filter FFT in complex128, the gather,
  the cross-lag / node log-sum-exp and the distance quadrature) -- the all-FP64
  oracle that gives the error of every result;
* precision='ref': the filter in complex64 with float32 trajectories, exactly as
  the reference's CPU path does (exmarg/search/bank.py:56-78), the rest as the
  reference (float64 gather arithmetic over float32 inputs).

Parity of this restatement with the reference itself is pinned by
tests/test_oracle_golden.py against vectors produced by running the reference's
own CPU code (tests/golden/make_golden.py).
"""

import ctypes
import os

import numpy as np

from . import build_oracle

NPHI = 96
_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        lib = ctypes.CDLL(build_oracle.build())
        P = ctypes.c_void_p
        lib.oracle_gather.argtypes = [ctypes.c_int, P, P, P, P, ctypes.c_int, ctypes.c_int, P, P, P,
                                      ctypes.c_int, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_int, P, P, ctypes.c_int, P]
        lib.oracle_gather.restype = ctypes.c_int
        lib.oracle_num_threads.restype = ctypes.c_int
        lib.oracle_gen_node.argtypes = [P, P, P, P, ctypes.c_float, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int, ctypes.c_int]
        lib.oracle_gen_node.restype = None
        _LIB = lib
    return _LIB


def num_threads():
    return int(_lib().oracle_num_threads())


def gen_tables(spec, s_nodes, seed, factors=None):
    """every node table of the seeded synthetic store, generated in C over the host cores
    (bit-identical to exmarg_b200.synth.gen_table_node)"""
    M, P, Q, S = factors if factors is not None else spec.factors(s_nodes)
    M, P, Q = (np.ascontiguousarray(x, np.float32) for x in (M, P, Q))
    out = []
    for k in range(len(s_nodes)):
        T = np.empty(spec.shape, np.float32)
        _lib().oracle_gen_node(T.ctypes.data, M.ctypes.data, P.ctypes.data, Q.ctypes.data, float(S[k]), int(seed),
                               k, spec.ntau, spec.nphif, spec.nb, spec.nd)
        out.append(T)
    return out


# ----------------------------------------------------------------------------- segments

def read_segments(segments, rows=None):
    """exmarg/search/segments.py:11-37: d_H, d_L as complex128, sig2_H/L float64"""
    z = np.load(segments) if isinstance(segments, (str, bytes, os.PathLike)) else segments
    n = np.asarray(z["d_H"]).shape[0]
    rows = np.arange(n) if rows is None else np.asarray(rows, int)
    out = {"rows": rows, "f": np.asarray(z["f"], float), "nu": np.asarray(z["nu"], np.int64),
           "T": float(z["T"]), "fmin": float(z["fmin"]), "fmax": float(z["fmax"])}
    for I in "HL":
        out["d_" + I] = np.asarray(z["d_" + I])[rows].astype(complex)
        key = "sig2_" + I if "sig2_" + I in z else "sig2"
        out["sig2_" + I] = np.asarray(z[key], float)
    return out


# ----------------------------------------------------------------------------- filter

def trajectories(W, d, sig2, lo, n_time, precision="fp64"):
    """exmarg/search/bank.py:56-78: z_I = FFT(pad(W conj(d_I) / sig2_I)), ln|z| and arg z.

    W (n_template, n_freq) complex; returns dict lqH, phH, lqL, phL (n_template, n_time),
    float64 for 'fp64', float32 (complex64 FFT) for 'ref'."""
    out = {}
    for I in "HL":
        if precision == "ref":
            w = np.ascontiguousarray(np.conj(d[I]) / sig2[I], np.complex64)
            pad = np.zeros((W.shape[0], n_time), np.complex64)
            pad[:, lo:lo + W.shape[1]] = np.asarray(W, np.complex64) * w[None, :]
            z = np.fft.fft(pad, axis=-1)
            lq = 0.5 * np.log(np.maximum(z.real ** 2 + z.imag ** 2, 1e-38))
            ph = np.arctan2(z.imag, z.real)
        else:
            w = np.conj(d[I]) / sig2[I]
            pad = np.zeros((W.shape[0], n_time), np.complex128)
            pad[:, lo:lo + W.shape[1]] = np.asarray(W, np.complex128) * w[None, :]
            z = np.fft.fft(pad, axis=-1)
            lq = 0.5 * np.log(np.maximum(z.real ** 2 + z.imag ** 2, 1e-38))
            ph = np.arctan2(z.imag, z.real)
        out["lq" + I], out["ph" + I] = lq, ph
    return out


# ----------------------------------------------------------------------------- time selection

def select_times(traj, tau_idx, n_loud, n_random, seed, bank_rows=None, n_bank=None):
    """exmarg/search/gather.py:374-420: the n_loud loudest times by |z_L|^2 + max_tau |z_H(t+tau)|^2,
    plus n_random host-RNG draws from the rest with log weight ln((n_time - n_loud) / n_random);
    returns (sel int32, lw float32), (n_template, n_loud + n_random), sorted by time.

    bank_rows / n_bank: the trajectories are rows bank_rows of an n_bank-template bank; the draws
    are then the rows of the whole bank's (n_bank, n_random) draw, as the reference takes them."""
    K, S = int(n_loud), int(n_random)
    lqH, lqL = traj["lqH"], traj["lqL"]
    nm, nt = lqH.shape
    lags = np.asarray(tau_idx).ravel().astype(int)
    lo, hi = int(lags.min()), int(lags.max())
    if not np.array_equal(np.sort(lags), np.arange(lo, hi + 1)):
        raise ValueError("lags are not contiguous")
    if bank_rows is None:
        pick = np.random.default_rng(seed).integers(0, nt - K, size=(nm, S))
    else:
        pick = np.random.default_rng(seed).integers(0, nt - K, size=(int(n_bank), S))[np.asarray(bank_rows)]
    # the sliding maximum over lags lo..hi (a direct window maximum; ln|z| is monotone in |z|^2)
    mx = np.full_like(lqH, -np.inf)
    for tau in range(lo, hi + 1):
        mx = np.maximum(mx, np.roll(lqH, -tau, axis=1))
    score = np.exp(2.0 * lqL) + np.exp(2.0 * mx)
    sel = np.empty((nm, K + S), np.int64)
    lw = np.zeros((nm, K + S), np.float32)
    lw[:, K:] = np.log((nt - K) / S)
    for m in range(nm):
        top = np.argpartition(-score[m], K)[:K]
        rest = np.ones(nt, bool)
        rest[top] = False
        rest = np.nonzero(rest)[0]
        sel[m] = np.concatenate([top, rest[pick[m]]])
    order = np.argsort(sel, axis=1, kind="stable")
    return (np.take_along_axis(sel, order, axis=1).astype(np.int32),
            np.take_along_axis(lw, order, axis=1))


# ----------------------------------------------------------------------------- gather

def gather(traj, tables, mass_ids, lna, tab_ids, beta, delta, tau_idx, times=None):
    """exmarg/search/gather.py:114-140 (gather_cpu contract): (NS, nsel) float64 ln Lambda.
    float32 trajectories get the reference's float32 phase difference (gather.py:54)."""
    lib = _lib()
    phase_f32 = int(np.asarray(traj["phH"]).dtype == np.float32)
    lqH, phH, lqL, phL = (np.ascontiguousarray(traj[k], np.float64) for k in ("lqH", "phH", "lqL", "phL"))
    nm, nt = lqH.shape
    ids = np.ascontiguousarray(mass_ids, np.int64)
    tab = np.ascontiguousarray(tab_ids, np.int64)
    lna = np.ascontiguousarray(lna, np.float64)
    nsel, ns = tab.shape
    T = [np.ascontiguousarray(t, np.float32) for t in tables]
    ptrs = (ctypes.c_void_p * len(T))(*[t.ctypes.data for t in T])
    ntau, nphif, nb, nd = T[0].shape
    tau = np.ascontiguousarray(tau_idx, np.int64).ravel()
    if times is not None:
        sel = np.ascontiguousarray(times[0], np.int32)
        lw = np.ascontiguousarray(times[1], np.float32)
        nwalk, psel, plw = sel.shape[1], sel.ctypes.data, lw.ctypes.data
    else:
        nwalk, psel, plw = 0, None, None
    out = np.empty((ns, nsel), np.float64)
    rc = lib.oracle_gather(nt, lqH.ctypes.data, phH.ctypes.data, lqL.ctypes.data, phL.ctypes.data,
                           nsel, ns, ids.ctypes.data, tab.ctypes.data, lna.ctypes.data,
                           ntau, tau.ctypes.data, ptrs, nphif, nb, nd,
                           float(beta[0]), float(beta[1] - beta[0]), float(delta[0]), float(delta[1] - delta[0]),
                           nwalk, psel, plw, phase_f32, out.ctypes.data)
    if rc:
        raise MemoryError("oracle gather: allocation failed")
    return out


# ----------------------------------------------------------------------------- node geometry, priors

def node_geometry(s, alpha_lo, alpha_hi, u, ymin):
    """exmarg/search/pe.py:58-84: valid (node, template) pairs, ln a, y, boundary node and its ln a"""
    nn, nm = s.size, u.size
    valid = np.zeros((nn, nm), bool)
    lna = np.zeros((nn, nm))
    y = np.zeros((nn + 1, nm))
    bnode = np.full(nm, -1)
    blna = np.zeros(nm)
    for k in range(nn):
        alo = min(alpha_lo[k], ymin * ymin)
        a = s[k] / u
        o = (np.sqrt(a) >= ymin) & (a > alo) & (a < alpha_hi[k])
        valid[k] = o
        lna[k][o] = np.log(a[o])
        y[k] = np.where(o, np.sqrt(a), 0.0)
        s_prev = s[k - 1] if k > 0 else 0.0
        low = o & (s_prev / u <= alo)
        a_b = float(alo) * (1.0 + 1e-9)
        bnode[low] = k
        blna[low] = np.log(a_b)
        y[nn][low] = np.sqrt(a_b)
    return valid, lna, y, bnode, blna


def distance_weights(y, prior, ymin, density=None, quadrature="reference"):
    """exmarg/search/pe.py:260-286: ln of the weights that integrate the distance prior against
    a likelihood ratio linear in ln y between the points y (ascending).  prior 'volume' is exact;
    'madau-dickinson' uses the trapezoid rule on 401 points per interval over density (lny, p_lny).
    quadrature='gl64': both by 64-point Gauss-Legendre in ln y on every interval (numpy's leggauss)."""
    x = np.log(y)
    w = np.zeros_like(x)
    gx, gw = np.polynomial.legendre.leggauss(64)
    for i in range(x.size - 1):
        a, b = x[i], x[i + 1]
        h = b - a
        if quadrature == "gl64":
            t = 0.5 * (a + b) + 0.5 * h * gx
            f = 3.0 * ymin ** 3 * np.exp(-3.0 * t) if prior == "volume" else \
                np.interp(t, density[0], density[1], left=0.0, right=0.0)
            w[i] += 0.5 * np.sum(gw * f * (b - t))
            w[i + 1] += 0.5 * np.sum(gw * f * (t - a))
        elif prior == "volume":
            c, k = 3.0 * ymin ** 3, 3.0
            ea, eb = np.exp(-k * a), np.exp(-k * b)
            I0 = (ea - eb) / k
            I1 = (a * ea - b * eb) / k + (ea - eb) / k ** 2
            w[i] += c * (b * I0 - I1) / h
            w[i + 1] += c * (I1 - a * I0) / h
        else:
            t = np.linspace(a, b, 401)
            f = np.interp(t, density[0], density[1], left=0.0, right=0.0)
            w[i] += np.trapezoid(f * (b - t) / h, t)
            w[i + 1] += np.trapezoid(f * (t - a) / h, t)
    with np.errstate(divide="ignore"):
        return np.log(w)


def ln_weights(yN, prior, ymin, density=None, quadrature="reference"):
    """exmarg/search/pe.py:321-327: lnW (n_node + 1, n_template), -inf where a template has no point"""
    lnW = np.full(yN.shape, -np.inf)
    for m in range(yN.shape[1]):
        pts = np.nonzero(yN[:, m] > 0)[0]
        if pts.size < 2:
            raise ValueError("template %d reaches fewer than two store nodes" % m)
        order = pts[np.argsort(yN[pts, m])]
        lnW[order, m] = distance_weights(yN[order, m], prior, ymin, density, quadrature)
    return lnW


def cell_weights(M, q, chi):
    """exmarg/search/pe.py:338-343: normalised product of the spacings of the distinct values per axis"""
    cell = np.ones(M.size)
    for ax in (M, q, chi):
        vals = np.unique(ax)
        if vals.size > 1:
            cell *= np.gradient(vals)[np.searchsorted(vals, ax)]
    return cell / cell.sum()


def log_mean(lam, w):
    """exmarg/search/pe.py:135-142"""
    fin = np.isfinite(lam) & (w > 0)
    if not fin.any():
        return -np.inf
    mx = np.where(fin, lam, -np.inf).max()
    return float(mx + np.log(np.sum(np.where(fin, w * np.exp(np.where(fin, lam, mx) - mx), 0.0))))


# ----------------------------------------------------------------------------- pe_intrinsic

def node_values(traj, store, geometry, groups, times):
    """exmarg/search/pe.py:168-200 for one segment: (n_node + 1, n_template), row n_node the boundary"""
    valid, lna, _, bnode, blna = geometry
    nn = store.s.size
    nm = valid.shape[1]
    lamN = np.full((nn + 1, nm), -np.inf)
    for ks in groups:
        k0 = ks[0]
        tab = [store.tables[k] for k in ks]
        beta, delta = store.beta[k0], store.delta[k0]
        ok = valid[ks]
        ids = np.nonzero(ok.any(axis=0))[0]
        lnaM = np.where(ok[:, ids], lna[ks][:, ids], 0.0).T
        tid = np.tile(np.arange(len(ks)), (ids.size, 1))
        bids = np.nonzero((bnode >= k0) & (bnode <= ks[-1]))[0]
        if ids.size:
            val = gather(traj, tab, ids, lnaM, tid, beta, delta, store.tau_idx, times)
            for i, k in enumerate(ks):
                keep = ok[i][ids]
                lamN[k, ids[keep]] = val[i][keep]
        if bids.size:
            val = gather(traj, tab, bids, blna[bids][:, None], (bnode[bids] - k0)[:, None], beta, delta,
                         store.tau_idx, times)
            lamN[nn, bids] = val[0]
    return lamN


def pe_intrinsic(seg, W, u, M, q, chi, lo, n_time, store, prior="volume", ymin=0.1267, nodes_per_launch=6,
                 n_loud=1024, n_random=1024, seed=0, precision="fp64", density=None, times=None,
                 return_parts=False, bank_rows=None, n_bank=None, quadrature="reference"):
    """exmarg/search/pe.py:289-346 for the segments of seg (read_segments output).
    quadrature='gl64': the distance prior by 64-point Gauss-Legendre (distance_weights).

    W (n_template, n_freq) complex template factors, u (n_template,) their powers.
    times: optional list (one per segment) of (sel, lw) to use instead of select_times
    (so that a numerical comparison is made on the same visited times).
    bank_rows / n_bank: W, u, M, q, chi are rows bank_rows of an n_bank-template bank (a
    template sample); the random draws are taken as for the whole bank (ln_b is then over
    the sample only).
    returns dict ln_lambda (n_seg, n_template), ln_b (n_seg,) [, parts]"""
    geometry = node_geometry(store.s, store.alpha_lo, store.alpha_hi, u, ymin)
    yN = geometry[2]
    nn = store.s.size
    groups = [list(range(g, min(g + nodes_per_launch, nn))) for g in range(0, nn, nodes_per_launch)]
    lnW = ln_weights(yN, prior, ymin, density, quadrature)
    nseg = seg["rows"].size
    out = np.full((nseg, u.size), -np.inf)
    parts = []
    for e in range(nseg):
        traj = trajectories(W, {I: seg["d_" + I][e] for I in "HL"}, {I: seg["sig2_" + I] for I in "HL"},
                            lo, n_time, precision)
        if times is not None:
            tm = times[e]
        elif n_loud > 0:
            tm = select_times(traj, store.tau_idx, n_loud, n_random, seed + int(seg["rows"][e]), bank_rows, n_bank)
        else:
            tm = None
        lamN = node_values(traj, store, geometry, groups, tm)
        v = lnW + lamN
        mx = v.max(axis=0)
        out[e] = mx + np.log(np.exp(v - mx[None, :]).sum(axis=0))
        if return_parts:
            parts.append(dict(lamN=lamN, times=tm, traj=traj))
    w = cell_weights(M, q, chi)
    ln_b = np.array([log_mean(L, w) for L in out])
    res = dict(ln_lambda=out, ln_b=ln_b, lnW=lnW)
    if return_parts:
        res["parts"] = parts
    return res


# ----------------------------------------------------------------------------- pe_redshift

def source_frame(lamN, yN, Mdet, yq, m1, z):
    """exmarg/search/pe.py:87-132 (_to_source_frame, numpy): node values (n_node + 1, n_template) ->
    ln Lambda (nm1, nz): linear in y per template between its finite node values, then linear in
    M_det = 2 m1 (1 + z) per z between the finite templates"""
    L, Y = np.asarray(lamN, float), np.asarray(yN, float)
    ok = np.isfinite(L) & (Y > 0)
    Yk = np.where(ok, Y, np.inf)
    order = np.argsort(Yk, axis=0, kind="stable")
    Ys = np.take_along_axis(Yk, order, axis=0)
    Ls = np.take_along_axis(L, order, axis=0)
    n = ok.sum(axis=0)
    nm = Ys.shape[1]
    cols = np.arange(nm)[None, :]
    j = (Ys[:, None, :] <= np.asarray(yq)[None, :, None]).sum(axis=0) - 1
    lo = np.clip(j, 0, np.maximum(n - 2, 0)[None, :])
    hi = np.minimum(lo + 1, np.maximum(n - 1, 0)[None, :])
    y0, y1, v0, v1 = Ys[lo, cols], Ys[hi, cols], Ls[lo, cols], Ls[hi, cols]
    yq_ = np.asarray(yq)[:, None]
    with np.errstate(invalid="ignore", divide="ignore"):
        t = np.where(y1 > y0, (yq_ - y0) / np.where(y1 > y0, y1 - y0, 1.0), 1.0)
        ylast = Ys[np.maximum(n - 1, 0), np.arange(nm)][None, :]
        inside = (n[None, :] >= 2) & (yq_ >= Ys[0][None, :]) & (yq_ <= ylast)
        surf = np.where(inside, v0 + t * (v1 - v0), -np.inf)
    M = np.asarray(Mdet, float)
    good = np.isfinite(surf)
    rank = np.cumsum(good, axis=1)
    ngood = rank[:, -1]
    G = np.zeros(surf.shape, np.int64)
    iz, im = np.nonzero(good)
    G[iz, rank[iz, im] - 1] = im
    Md = 2.0 * np.asarray(m1)[:, None] * (1.0 + np.asarray(z))[None, :]
    p = np.searchsorted(M, Md.ravel()).reshape(Md.shape)
    zi = np.arange(len(z))[None, :]
    below = np.where(p > 0, rank[zi, np.maximum(p - 1, 0)], 0)
    lo = G[zi, np.clip(below - 1, 0, None)]
    hi = G[zi, np.minimum(below, np.maximum(ngood - 1, 0)[None, :])]
    lo = np.where(below >= 1, lo, hi)
    m0, m1_ = M[lo], M[hi]
    w0, w1 = surf[zi, lo], surf[zi, hi]
    with np.errstate(invalid="ignore", divide="ignore"):
        t = np.where(m1_ > m0, (Md - m0) / np.where(m1_ > m0, m1_ - m0, 1.0), 0.0)
        first = M[G[:, 0]][None, :]
        last = M[G[zi[0], np.maximum(ngood - 1, 0)]][None, :]
        inb = (ngood[None, :] >= 2) & (Md >= first) & (Md <= last)
        return np.where(inb, w0 + t * (w1 - w0), -np.inf)


def redshift_weights(m1, z, dl, mdet_range):
    """exmarg/search/pe.py:249-254: prior weights on the (m1, z) cells, uniform in M_det on mdet_range
    and proportional to (1 + z) D_L^2 dD_L/dz; normalised"""
    lnp = np.log(np.maximum((1.0 + z) * dl ** 2 * np.gradient(dl, z), 1e-300))
    Md = 2.0 * m1[:, None] * (1.0 + z[None, :])
    inside = (Md >= mdet_range[0]) & (Md <= mdet_range[1])
    w = np.where(inside, np.exp(lnp)[None, :], 0.0) * np.gradient(m1)[:, None] * np.gradient(z)[None, :]
    return w / w.sum()


def pe_redshift(seg, W, u, M, lo, n_time, store, dl_of_z, zmax=8.0, nz=1600, m1_range=(3.0, 150.0), nm1=1600,
                ymin=0.1267, nodes_per_launch=6, mdet_range=(10.0, 500.0), n_loud=1024, n_random=1024, seed=0,
                precision="ref"):
    """exmarg/search/pe.py:203-257 for the segments of seg (read_segments output): ln Lambda (n_seg, nm1, nz)
    on z = linspace(0.02, zmax, nz), m1 = geomspace(*m1_range, nm1), and ln B; dl_of_z is the distance
    function (the reference's is astropy's Planck18)"""
    from exmarg_b200.segments import D0
    z = np.linspace(0.02, zmax, int(nz))
    m1 = np.geomspace(m1_range[0], m1_range[1], int(nm1))
    dl = dl_of_z(z)
    yq = D0 / dl
    geometry = node_geometry(store.s, store.alpha_lo, store.alpha_hi, u, ymin)
    nn = store.s.size
    groups = [list(range(g, min(g + nodes_per_launch, nn))) for g in range(0, nn, nodes_per_launch)]
    out = np.full((seg["rows"].size, m1.size, z.size), -np.inf)
    for e in range(seg["rows"].size):
        traj = trajectories(W, {I: seg["d_" + I][e] for I in "HL"}, {I: seg["sig2_" + I] for I in "HL"}, lo,
                            n_time, precision)
        tm = select_times(traj, store.tau_idx, n_loud, n_random, seed + int(seg["rows"][e])) if n_loud > 0 else None
        lamN = node_values(traj, store, geometry, groups, tm)
        out[e] = source_frame(lamN, geometry[2], M, yq, m1, z)
    w = redshift_weights(m1, z, dl, mdet_range)
    ln_b = np.array([log_mean(L, w) for L in out])
    return dict(m1=m1, z=z, ln_lambda=out, ln_b=ln_b)


# ----------------------------------------------------------------------------- table build, stage 3

def bd_tables(col, row, lnq, beta, ladder):
    """scripts/build_tables/build_bd.py:53-77: T_nm[tau, phi, b, d] = log sum_{n <= nm} exp(n beta_b + g_n(Delta_d))
    for each truncation order nm, float64 arithmetic rounded to float32.

    col, row: (orders, lags, nq, nphif) -- lnK on the last column (q2 = q_last) and the last row (q1 = q_last);
    g_n on Delta <= 0 is col - 2n ln q_last (Delta ascending with q1), on Delta > 0 row - 2n ln q2 (q2 descending)."""
    col = np.asarray(col, np.float64)
    row = np.asarray(row, np.float64)
    lnq = np.asarray(lnq, np.float64)
    beta = np.asarray(beta, np.float64)
    nord, ntau, nq, nphif = col.shape
    n = np.arange(nord, dtype=np.float64)
    two_n = 2.0 * n
    out = {nm: np.empty((ntau, nphif, beta.size, 2 * nq - 1), np.float32) for nm in ladder}
    nbeta = n[:, None] * beta[None, :]                                   # (orders, nb)
    for t in range(ntau):
        lo = col[:, t] - (two_n * lnq[-1])[:, None, None]               # (orders, nq, nphif), q1 ascending
        hi = row[:, t] - two_n[:, None, None] * lnq[None, :, None]      # q2 ascending
        g = np.concatenate([lo, hi[:, -2::-1]], axis=1)                 # (orders, 2 nq - 1, nphif)
        for p in range(nphif):
            E = nbeta[:, :, None] + g[None, :, :, p].transpose(1, 0, 2)   # (orders, nb, nd)
            for nm in ladder:
                mx = E[:nm + 1].max(axis=0)
                tot = np.zeros_like(mx)
                for k in range(nm + 1):                                  # in order of n
                    tot += np.exp(E[k] - mx)
                out[nm][t, p] = (mx + np.log(tot)).astype(np.float32)
    return out


# ----------------------------------------------------------------------------- table build, stage 1

def w_table_s(s_nodes, n_max, nside, n_tau, pix2ang, rounding="numpy"):
    """scripts/build_tables/w_gpu.py:104-182 (the GORFs at fixed distance), float64 numpy, pixel by pixel:
    responses in float32 as the reference forms them (complex64), |R|^2 and arg R in float32, then ladders,
    damping and the per-key quadrature sums in float64, the linear delay deposit and the s^n 2^n / n! scale.
    rounding: 'numpy' takes |R| and arg R from numpy's float32 abs and angle (as the reference run on numpy
    does); 'correct' rounds them to float32 from float64 (the float32 functions of numpy, CUDA and a
    correctly rounded evaluation differ in the last bit).
    Returns tau, W (n_nodes, n_tau, n_keys) float64 over the keys (n, a, b), b <= a, in order."""
    from scipy.special import gammaln
    from exmarg_b200 import wtable as wt
    s = np.atleast_1d(np.asarray(s_nodes, float))
    psi, cg, wq = wt.quadrature(n_max)
    tau = wt.tau_grid(n_tau)
    npix = 12 * nside * nside
    th, ph = pix2ang(nside, np.arange(npix))
    j0, w = wt.deposit(tau, th, ph, npix)
    ks = wt.keys(n_max)
    c2p, s2p = np.cos(2 * psi).astype(np.float32), np.sin(2 * psi).astype(np.float32)
    Ap, cgf = (0.5 * (1 + cg ** 2)).astype(np.float32), cg.astype(np.float32)
    Wraw = np.zeros((s.size, n_tau, len(ks)))
    for p in range(npix):
        R = []
        for I in "HL":
            fp, fx = wt.antenna(I, th[p:p + 1], ph[p:p + 1])
            fp, fx = np.float32(fp[0]), np.float32(fx[0])
            Fp = fp * c2p - fx * s2p
            Fx = fp * s2p + fx * c2p
            R.append((Ap[None, :] * Fp[:, None] + 1j * cgf[None, :] * Fx[:, None]).astype(np.complex64).ravel())
        if rounding == "correct":
            re = [r.real.astype(np.float64) for r in R]
            im = [r.imag.astype(np.float64) for r in R]
            mag = [np.sqrt(a * a + b * b).astype(np.float32) for a, b in zip(re, im)]
            ang = [np.arctan2(b, a).astype(np.float32) for a, b in zip(re, im)]
        else:
            mag = [np.abs(r) for r in R]
            ang = [np.angle(r) for r in R]
        S1, S2 = ((mg * mg).astype(np.float64) for mg in mag)
        dph = (ang[0] - ang[1]).astype(np.float64)
        m1, m2 = np.sqrt(S1 / 2.0), np.sqrt(S2 / 2.0)
        wqf = np.broadcast_to(wq[None, :], (psi.size, cg.size)).ravel()
        Bw = np.stack([np.exp(-(sj * S1 + sj * S2)) for sj in s]) * wqf[None, :]        # (nodes, Q)
        V = np.empty((s.size, len(ks)))
        for k, (n, a, b) in enumerate(ks):
            V[:, k] = (Bw * np.cos((a - b) * dph)[None, :]) @ (m1 ** (a + b) * m2 ** (2 * n - a - b))
        Wraw[:, j0[p]] += w[p, 0] * V
        Wraw[:, j0[p] + 1] += w[p, 1] * V
    n_key = np.array([k[0] for k in ks], float)
    scale = np.exp(np.minimum(n_key[None, :] * np.log(s)[:, None] - gammaln(n_key + 1.0)[None, :]
                              + n_key[None, :] * np.log(2.0), 700.0))
    return tau, Wraw * scale[:, None, :]


# ----------------------------------------------------------------------------- table build, stage 2

def k_order(n, s, keys, Wd, lnq, phi, pairs=None):
    """scripts/build_tables/build_k.py:59-82 for one order n: lnK_n (n_tau, n_pairs, n_phi) float32 on the
    (q1, q2) pairs given as index arrays (q1, q2) (default: the whole nq x nq grid, row-major), with the
    reference's grouping: per phase class m = a - b the sum over its (a, b) as one product of matrices, then
    the cosine sum over m."""
    from scipy.special import comb, gammaln
    nq = lnq.size
    if pairs is None:
        q1, q2 = (x.ravel() for x in np.meshgrid(np.arange(nq), np.arange(nq), indexing="ij"))
    else:
        q1, q2 = pairs
    l1, l2 = lnq[q1], lnq[q2]
    o_n = gammaln(n + 1.0) + n * np.log(s)
    g = 2.0 * n * np.maximum(l1, l2)
    rows = [(j, int(a), int(b)) for j, (nn, a, b) in enumerate(keys) if nn == n]
    ms = sorted({a - b for _, a, b in rows})
    C = np.empty((len(ms), Wd.shape[1] * l1.size))
    for i, m in enumerate(ms):
        sel = [(j, a, b) for j, a, b in rows if a - b == m]
        Wm = np.array([comb(n, a) * comb(n, b) * (2.0 if m else 1.0) * Wd[j] for j, a, b in sel])
        P = np.exp(np.stack([(a + b) * l1 + (2 * n - a - b) * l2 - g for _, a, b in sel]))
        C[i] = (Wm.T @ P).ravel()
    K = (C.T @ np.cos(np.outer(ms, phi))).reshape(Wd.shape[1], l1.size, phi.size)
    return (np.log(np.maximum(K, 1e-300)) + (g - o_n)[None, :, None]).astype(np.float32)


def k_edges(keys, Wd, s, n_max, lnq, nphi):
    """lnK's last column (q2 = q_last) and last row (q1 = q_last), (orders, lags, nq, nphi/2 + 1) float32 each"""
    nq = lnq.size
    phi = (np.arange(nphi) * (2 * np.pi / nphi))[:nphi // 2 + 1]
    last = np.full(nq, nq - 1)
    ar = np.arange(nq)
    col = np.stack([k_order(n, s, keys, Wd, lnq, phi, (ar, last)) for n in range(n_max + 1)]).transpose(0, 1, 2, 3)
    row = np.stack([k_order(n, s, keys, Wd, lnq, phi, (last, ar)) for n in range(n_max + 1)])
    return col, row
