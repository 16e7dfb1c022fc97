"""The offline table build, stages 2 and 3 (the contracts of scripts/build_tables/build_k.py and
build_bd.py): from a node's GORFs W (stage 1) through lnK_n(tau, q1, q2, phi) to its table
T[tau, phi+, beta, Delta] (the bd_*.npz that load_redshift_store reads), on the B200.

build_node_from_w goes from W to the table without the 49 GB lnK of stage 2: the table needs lnK only on
the last column and last row of the (q1, q2) grid, and exm_k_edges computes just those (with the
reference's grouping: per phase class m the sum over its (a, b), then the cosine sum over m).

Only the last column and the last row of each (q1, q2) block of lnK enter the table (every order is
homogeneous in (q1, q2)), so build_node reads just those slices of the memory-mapped lnK and
exm_bd_build forms the log-sum over the orders on the device in float64 (one pass for every
truncation order of the ladder, as BD_NMAX_LADDER asks the reference).
"""

import os
import time

import numpy as np

from . import _lib

ALPHA = np.geomspace(0.16, 4.0e4, 30)     # the amplitude axis; it sets the range of beta (build_bd.py:26)


def bd_grid(lnq, alpha=ALPHA):
    """(beta, delta) of a node's table from its magnitude grid (build_bd.py:56-63)"""
    lnq = np.asarray(lnq, np.float64)
    last = lnq.size - 1
    dlq = float(lnq[1] - lnq[0])
    delta = np.concatenate([lnq - lnq[last], (lnq[last] - lnq)[::-1][1:]])
    dbeta = 2.0 * dlq
    b_lo = np.log(alpha[0]) + 2.0 * lnq[0]
    b_hi = np.log(alpha[-1]) + 2.0 * lnq[-1]
    nb = int(np.ceil((b_hi - b_lo) / dbeta)) + 1
    return b_lo + dbeta * np.arange(nb), delta


def lnk_edges(A):
    """(col, row): the last column A[:, :, :, -1, :nphif] and last row A[:, :, -1, :, :nphif] of
    stage 2's lnK (orders, lags, nq, nq, nphi), float32"""
    nphif = A.shape[4] // 2 + 1
    col = np.ascontiguousarray(A[:, :, :, -1, :nphif], np.float32)
    row = np.ascontiguousarray(A[:, :, -1, :, :nphif], np.float32)
    return col, row


def bd_tables(col, row, lnq, ladder=None, device=0, ctx=None):
    """{n_max: T (lags, nphif, nb, 2 nq - 1) float32}, beta, delta, stats for the truncation orders
    in ladder (default: every order); raises FloatingPointError on a non-finite entry as the
    reference does"""
    nord = np.shape(col)[0]
    ladder = [nord - 1] if ladder is None else [int(v) for v in ladder]
    if max(ladder) > nord - 1:
        raise ValueError("a truncation order exceeds the orders of lnK")
    beta, delta = bd_grid(lnq)
    ctx = ctx or _lib.context(device)
    T, bad, ms = ctx.bd_build(col, row, lnq, beta, ladder)
    if bad:
        raise FloatingPointError("table has non-finite entries at n_max=%d" % ladder[0])
    return {nm: T[i] for i, nm in enumerate(ladder)}, beta, delta, {"kernel_ms": ms[0], "ms": ms[1]}


# the data delay grid of stage 2 (build_k.py:31-34): T = 4 s at f_max = 512 Hz, step 1 / (8 f_max)
K_T, K_FMAX = 4.0, 512.0
K_QMAX, K_QSPAN, K_NQ, K_NPHI = 100.0, 2000.0, 110, 96


def rebin(tau_fine, W_fine, tau_new):
    """W (keys, fine delays) summed into the bins of tau_new, each fine delay to the nearest new delay
    (bin edges half-way, the end bins open); sums kept exactly (exmarg/tables.py:253-268)"""
    order = np.argsort(tau_new)
    ts = np.asarray(tau_new, np.float64)[order]
    edges = np.concatenate([[ts[0] - 0.5 * (ts[1] - ts[0])], 0.5 * (ts[1:] + ts[:-1]), [ts[-1] + 0.5 * (ts[-1] - ts[-2])]])
    idx = np.clip(np.searchsorted(edges, tau_fine) - 1, 0, ts.size - 1)
    W_fine = np.asarray(W_fine, np.float64)
    acc = np.zeros((W_fine.shape[0], ts.size))
    for f in range(W_fine.shape[1]):             # in order of the fine delays, as the reference accumulates
        acc[:, idx[f]] += W_fine[:, f]
    out = np.empty_like(acc)
    out[:, order] = acc
    return out


def load_w_node(stem, T=K_T, fmax=K_FMAX):
    """a stage-1 node (<stem>.W.npy, .meta.npz) on the data delays: keys (n, a, b <= a), W (keys, lags),
    tau_idx (build_k.py:37-49)"""
    m = np.load(stem + ".meta.npz")
    Wa = np.load(stem + ".W.npy").astype(np.float64)
    tau_f = m["tau"]
    n_time = 8 * int(fmax * T)
    tau_all = np.fft.fftfreq(n_time) * T
    t_step = T / n_time
    keep = np.abs(tau_all) <= 1.05 * np.abs(tau_f).max()
    tau_idx = np.rint(tau_all[keep] / t_step).astype(int)
    keys = np.asarray(m["keys"]).astype(np.int64)
    Wd = rebin(tau_f, Wa, tau_all[keep])
    order = np.lexsort((keys[:, 2], keys[:, 1], keys[:, 0]))
    return keys[order], Wd[order], tau_idx, float(m["s_node"]), int(m["n_max"])


def k_inputs(keys, s, n_max, lnq, nphi=K_NPHI):
    """coeff per key C(n,a) C(n,b) (x2 for a > b), gmo per order 2n ln q_last - ln(n! s^n), cos(m phi_p) on the
    first nphi/2 + 1 phases (build_k.py:59-82)"""
    from scipy.special import comb, gammaln
    n, a, b = keys[:, 0], keys[:, 1], keys[:, 2]
    coeff = comb(n, a) * comb(n, b) * np.where(a != b, 2.0, 1.0)
    orders = np.arange(n_max + 1, dtype=np.float64)
    gmo = 2.0 * orders * lnq[-1] - (gammaln(orders + 1.0) + orders * np.log(s))
    phi_g = np.arange(nphi) * (2 * np.pi / nphi)
    cosm = np.cos(np.outer(np.arange(n_max + 1), phi_g))[:, :nphi // 2 + 1]
    return coeff, gmo, cosm


def build_node_from_w(stem_w, base, nq=K_NQ, nphi=K_NPHI, ladder=None, device=0, ctx=None):
    """stages 2 and 3 for one node: <stem_w>.W.npy / .meta.npz (build_w.py's output) -> <base>/bd_n<n_max>_s<s>.npz
    (and the truncated tables of ladder next to it), with only the lnK edges formed; returns the files written"""
    meta = np.load(stem_w + ".meta.npz")
    s, n_max = float(meta["s_node"]), int(meta["n_max"])
    ladder = [n_max] if ladder is None else [int(v) for v in ladder]
    if max(ladder) > n_max:
        raise ValueError("a truncation order exceeds the node's n_max")
    outs = {nm: os.path.join(out_dir(base, nm, n_max), "bd_n%03d_s%09.3f.npz" % (nm, s)) for nm in ladder}
    todo = [nm for nm in ladder if not os.path.exists(outs[nm])]   # tables already written are skipped
    if not todo:
        return []
    keys, Wd, tau_idx, s, n_max = load_w_node(stem_w)
    lnq = np.log(np.geomspace(K_QMAX / K_QSPAN, K_QMAX, nq))
    coeff, gmo, cosm = k_inputs(keys, s, n_max, lnq, nphi)
    ctx = ctx or _lib.context(device)
    col, row, _ = ctx.k_edges(n_max, Wd, coeff, lnq, gmo, cosm)
    Ts, beta, delta, _ = bd_tables(col, row, lnq, todo, ctx=ctx)
    for nm in todo:
        os.makedirs(os.path.dirname(outs[nm]), exist_ok=True)
        np.savez(outs[nm], T=Ts[nm], beta=beta, delta=delta, tau_idx=tau_idx, lnq=lnq, alpha=ALPHA, s_node=s, u_node=s,
                 n_max=nm, nphif=col.shape[3], norm="taylor_off1")
    return [outs[nm] for nm in todo]


def out_dir(base, nmax, nmax_full):
    """the full order in base, the truncated tables next to it (build_bd.py:30-32)"""
    return base if nmax == nmax_full else "%s_n%03d" % (base, nmax)


def build_node(stem, base, ladder=None, device=0):
    """one node: <stem>.meta.npz + <stem>.lnK.npy -> <base>/bd_n<order>_s<s>.npz (and the truncated
    tables of ladder, default BD_NMAX_LADDER, next to it); tables already written are skipped
    (build_bd.py:35-87).  Returns the files written."""
    meta = np.load(stem + ".meta.npz")
    s = float(meta["s_node"])
    lnq = meta["lnq"].astype(np.float64)
    tau_idx = meta["tau_idx"]
    nmax_full = int(os.path.basename(stem).split("_n")[1].split("_")[0])
    if ladder is None:
        env = os.environ.get("BD_NMAX_LADDER", "").strip()
        ladder = [int(v) for v in env.split(",")] if env else [nmax_full]
    if max(ladder) > nmax_full:
        raise ValueError("a truncation order exceeds the node's n_max")
    outs = {nm: os.path.join(out_dir(base, nm, nmax_full), "bd_n%03d_s%09.3f.npz" % (nm, s)) for nm in ladder}
    for d in {os.path.dirname(v) for v in outs.values()}:
        os.makedirs(d, exist_ok=True)
    todo = [nm for nm in ladder if not os.path.exists(outs[nm])]
    if not todo:
        return []
    t0 = time.time()
    A = np.load(stem + ".lnK.npy", mmap_mode="r")
    col, row = lnk_edges(A)
    Ts, beta, delta, _ = bd_tables(col, row, lnq, todo, device)
    nphif = col.shape[3]
    for nm in todo:
        np.savez(outs[nm], T=Ts[nm], beta=beta, delta=delta, tau_idx=tau_idx, lnq=lnq, alpha=ALPHA, s_node=s,
                 u_node=s, n_max=nm, nphif=nphif, norm="taylor_off1")
    print("s=%g done: %d orders %s in %.1f s" % (s, len(todo), todo, time.time() - t0), flush=True)
    return [outs[nm] for nm in todo]


def node_stems(directory, prefix, suffix):
    """the stems <directory>/<prefix>n<order>_s<s> of the files <stem><suffix>, in ascending s"""
    import glob
    files = glob.glob(os.path.join(directory, prefix + "n*_s*" + suffix))
    stems = [f[:-len(suffix)] for f in files]
    return sorted(stems, key=lambda t: float(os.path.basename(t).split("_s")[-1]))


def main(argv=None):
    """python -m exmarg_b200.tables bd <k_dir> <out_dir> [node indices]     stage 3 from stage 2's lnK (build_bd.py)
    python -m exmarg_b200.tables from-w <w_dir> <out_dir> [node indices] stages 2 + 3 from stage 1's W
    Node indices count the input files in ascending s (default: all).  BD_NMAX_LADDER as build_bd.py reads it."""
    import argparse
    ap = argparse.ArgumentParser(prog="python -m exmarg_b200.tables", description=main.__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("mode", choices=("bd", "from-w"))
    ap.add_argument("in_dir")
    ap.add_argument("out_dir")
    ap.add_argument("nodes", nargs="*", type=int)
    ap.add_argument("--nq", type=int, default=K_NQ, help="from-w: magnitude points of stage 2 (build_k.py: 110)")
    ap.add_argument("--nphi", type=int, default=K_NPHI, help="from-w: phase points of stage 2 (build_k.py: 96)")
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    env = os.environ.get("BD_NMAX_LADDER", "").strip()
    ladder = [int(v) for v in env.split(",")] if env else None
    if args.mode == "bd":
        stems = node_stems(args.in_dir, "kstore_", ".meta.npz")
    else:
        stems = node_stems(args.in_dir, "sladder_", ".meta.npz")
    if not stems:
        raise SystemExit("no input nodes in %s" % args.in_dir)
    pick = args.nodes or list(range(len(stems)))
    for i in pick:
        if args.mode == "bd":
            build_node(stems[i], args.out_dir, ladder, args.device)
        else:
            t0 = time.time()
            files = build_node_from_w(stems[i], args.out_dir, nq=args.nq, nphi=args.nphi, ladder=ladder,
                                      device=args.device)
            print("%s: %d tables in %.1f s" % (os.path.basename(stems[i]), len(files), time.time() - t0), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
