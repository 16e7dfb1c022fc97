"""pe_intrinsic on the B200 (the contract of exmarg/search/pe.py:289-346).

Same signature and return value as the reference.  With a 'b200' bank the whole
analysis of every segment -- matched filter, time selection (with numpy's PCG64
draws reproduced on the device), the plane-staged table gather with its
log-sum-exp, the node and distance-prior log-sum-exp and ln B -- runs in
libexmarg_b200 on one context; only d_H, d_L go in and ln_lambda, ln_b come out.
chunk, nodes_per_launch, block and resident are accepted and have no effect: the
tables stay resident and the device path sizes its own launches.  With a 'cpu' or
'gpu' bank the call goes to the reference's exmarg.search.pe_intrinsic.
"""

import numpy as np

from . import _lib
from .priors import distance_density
from .segments import read_segments
from .store import upload_store


def _density_key(prior):
    """a content key for a tabulated density (lny, p_lny)"""
    a, b = (np.ascontiguousarray(x, np.float64) for x in prior)
    return ("tabulated", a.size, hash(a.tobytes()), hash(b.tobytes()))


def prepare(bank, store, prior="volume", ymin=0.1267):
    """make (store, bank, prior, ymin) current on the bank's context: tables resident, geometry and
    distance weights computed on the device (once; later calls with the same inputs reuse them)"""
    ctx = bank.ctx
    upload_store(store, ctx)
    bank.upload()
    key = (ctx.store_token, ctx.bank_token, prior if isinstance(prior, str) else _density_key(prior), float(ymin))
    if ctx.prep_token != key:
        density = distance_density(prior)
        if density is None:
            ctx.prepare(ymin, _lib.PRIOR_VOLUME)
        else:
            ctx.prepare(ymin, _lib.PRIOR_TABULATED, density)
        ctx.prep_token = key
    return ctx


def pe_intrinsic(segments, bank, store, rows=None, prior="volume", ymin=0.1267, chunk=4, nodes_per_launch=6,
                 block=256, resident=False, n_loud=1024, n_random=1024, seed=0):
    """ln Lambda of each template of the bank, the distance integrated over its prior.

    returns dict: M, q, chi, u (n_template,), ln_lambda (n_segment, n_template),
    ln_b (n_segment,), rows."""
    if getattr(bank, "device", None) in ("cpu", "gpu"):
        import exmarg.search as ref
        return ref.pe_intrinsic(segments, bank, store, rows=rows, prior=prior, ymin=ymin, chunk=chunk,
                                nodes_per_launch=nodes_per_launch, block=block, resident=resident, n_loud=n_loud,
                                n_random=n_random, seed=seed)
    if getattr(bank, "device", None) != "b200":
        raise ValueError("device must be 'cpu', 'gpu' or 'b200'")
    if int(nodes_per_launch) < 1 or int(chunk) < 1:
        raise ValueError("chunk and nodes_per_launch must be >= 1")
    seg = read_segments(segments, rows)
    ctx = prepare(bank, store, prior, ymin)
    seeds = seed + np.asarray(seg["rows"], np.int64)
    lnl, lnb = ctx.pe_intrinsic(seg["d_H"], seg["d_L"], seg["sig2_H"], seg["sig2_L"], seeds, n_loud, n_random)
    return dict(M=bank.M, q=bank.q, chi=bank.chi, u=bank.u, ln_lambda=lnl, ln_b=lnb, rows=seg["rows"])


def autotune(bank, store, segments, prior="volume", ymin=0.1267, n_loud=1024, n_random=1024, reps=2):
    """choose the plane gather's launch shape and templates per block for this bank and store: analyse
    the first segment once, then time every shape on it (CUDA events), then the block size at 50 / 150 /
    200% with the best shape; later calls on the context use the fastest.
    returns (chosen shape index, ms per launch: each shape, then each block size)"""
    pe_intrinsic(segments, bank, store, rows=[0], prior=prior, ymin=ymin, n_loud=n_loud, n_random=n_random)
    return bank.ctx.autotune(n_loud, n_random, reps)


def distance_weights(y, prior, ymin):
    """ln of the distance-prior weights of points y (ascending), exmarg/search/pe.py:260-286 (host, float64)"""
    density = distance_density(prior)
    x = np.log(y)
    w = np.zeros_like(x)
    for i in range(x.size - 1):
        a, b = x[i], x[i + 1]
        h = b - a
        if density is None:
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
