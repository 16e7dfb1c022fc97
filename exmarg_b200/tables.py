"""The offline table build, stage 3 (the contract of scripts/build_tables/build_bd.py): from stage 2's
lnK_n(tau, q1, q2, phi) of one node to its table T[tau, phi+, beta, Delta] (the bd_*.npz that
load_redshift_store reads), on the B200.

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
