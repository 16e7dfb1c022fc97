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

import json
import os

import numpy as np

from . import _lib
from .priors import distance_density
from .segments import read_segments
from .store import upload_store


def _density_key(prior):
    """a content key for a tabulated density (lny, p_lny)"""
    a, b = (np.ascontiguousarray(x, np.float64) for x in prior)
    return ("tabulated", a.size, hash(a.tobytes()), hash(b.tobytes()))


QUADRATURES = ("reference", "gl64")


def prepare(bank, store, prior="volume", ymin=0.1267, quadrature="reference"):
    """make (store, bank, prior, ymin) current on the bank's context: tables resident, geometry and
    distance weights computed on the device (once; later calls with the same inputs reuse them).
    quadrature: 'reference' integrates the distance prior as exmarg/search/pe.py:260-286 does (closed form
    for the volume prior, 401-point trapezoid per interval for a tabulated density); 'gl64' uses 64-point
    Gauss-Legendre in ln y on every interval for both"""
    if quadrature not in QUADRATURES:
        raise ValueError("quadrature must be 'reference' or 'gl64'")
    ctx = bank.ctx
    upload_store(store, ctx)
    bank.upload()
    key = (ctx.store_token, ctx.bank_token, prior if isinstance(prior, str) else _density_key(prior), float(ymin),
           quadrature)
    if ctx.prep_token != key:
        density = distance_density(prior)
        gl = quadrature == "gl64"
        if density is None:
            ctx.prepare(ymin, _lib.PRIOR_VOLUME, gl64=gl)
        else:
            ctx.prepare(ymin, _lib.PRIOR_TABULATED, density, gl64=gl)
        ctx.prep_token = key
    return ctx


def pe_intrinsic(segments, bank, store, rows=None, prior="volume", ymin=0.1267, chunk=4, nodes_per_launch=6,
                 block=256, resident=False, n_loud=1024, n_random=1024, seed=0, quadrature="reference",
                 filter_precision="reference"):
    """ln Lambda of each template of the bank, the distance integrated over its prior.
    quadrature ('b200' only): 'reference' (the reference's rules) or 'gl64' (see prepare).
    filter_precision ('b200' only): 'reference' -- ln|z| rounded to float32 as the reference's filter leaves it,
    so results follow the reference's; 'fp64' -- ln|z| kept to float64 precision, so results follow the
    float64 evaluation (at high SNR the reference's float32 rounding moves ln B by up to ~1e-4)

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
    ctx = prepare(bank, store, prior, ymin, quadrature)
    ctx.set_filter_precision(filter_precision)
    seeds = seed + np.asarray(seg["rows"], np.int64)
    apply_tuned(ctx, n_loud, n_random)
    lnl, lnb = ctx.pe_intrinsic(seg["d_H"], seg["d_L"], seg["sig2_H"], seg["sig2_L"], seeds, n_loud, n_random)
    return dict(M=bank.M, q=bank.q, chi=bank.chi, u=bank.u, ln_lambda=lnl, ln_b=lnb, rows=seg["rows"])


def autotune(bank, store, segments, prior="volume", ymin=0.1267, n_loud=1024, n_random=1024, reps=2, cache=True):
    """choose the plane gather's launch shape and templates per block for this bank and store: analyse
    the first segment once, then time every shape on it (CUDA events), then the block size at 50 / 150 /
    200% with the best shape; later calls on the context use the fastest.  With cache, the choice is
    also written to the autotune cache (tune_cache_path()), from which later processes take it for the
    same workload shape on the same device model without tuning.
    returns (chosen shape index, ms per launch: each shape, then each block size)"""
    pe_intrinsic(segments, bank, store, rows=[0], prior=prior, ymin=ymin, n_loud=n_loud, n_random=n_random)
    ctx = bank.ctx
    best, ms = ctx.autotune(n_loud, n_random, reps)
    if cache:
        record_tuned(ctx, n_loud, n_random, best, ctx.gather_chunk_pct, ms)
    return best, ms


# ----------------------------------------------------------------------------- autotune cache

def tune_cache_path():
    """EXMARG_B200_TUNE_CACHE, else ~/.cache/exmarg_b200/autotune.json"""
    p = os.environ.get("EXMARG_B200_TUNE_CACHE")
    return p if p else os.path.join(os.path.expanduser("~"), ".cache", "exmarg_b200", "autotune.json")


def tune_key(ctx, n_loud, n_random):
    """the workload shape the gather's best launch depends on, and the device model (its memory size)"""
    nn, ntau, nphif, nb, nd, dtype = ctx.store_shape
    return "dev%d|templates%d|n_time%d|nodes%d|lags%d|planes%d|nb%d|nd%d|dtype%d|walk%d" % (
        int(ctx.device_total) >> 30, ctx.nm, ctx.n_time, nn, ntau, nphif, nb, nd, dtype,
        (n_loud + n_random) if n_loud > 0 else ctx.n_time)


def _read_cache(path):
    try:
        with open(path) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def record_tuned(ctx, n_loud, n_random, shape, chunk_pct, ms=None):
    """write an autotune choice to the cache (a JSON object keyed by tune_key; written atomically)"""
    path = tune_cache_path()
    d = _read_cache(path)
    d[tune_key(ctx, n_loud, n_random)] = {"shape": int(shape), "chunk_pct": int(chunk_pct),
                                          "ms": [float(v) for v in np.asarray(ms if ms is not None else [])[:16]]}
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tmp = path + ".%d.tmp" % os.getpid()
    with open(tmp, "w") as fh:
        json.dump(d, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def apply_tuned(ctx, n_loud, n_random):
    """use the cached choice for this workload when the context has none of its own (autotune or
    set_gather_cfg); returns the entry applied or None.  Child contexts keep the launch their parent
    chose (the library copies it when they are made), so that served and plain results agree bitwise."""
    if ctx.gather_cfg is not None or getattr(ctx, "parent", None) is not None:
        return None
    if ctx.store_shape is None or ctx.nm is None:
        return None
    key = tune_key(ctx, n_loud, n_random)
    if getattr(ctx, "tune_looked_up", None) == key:   # looked up already for this workload: no entry
        return None
    ctx.tune_looked_up = key
    e = _read_cache(tune_cache_path()).get(key)
    if not e or not 0 <= int(e.get("shape", -1)) < len(_lib.GATHER_SHAPES):
        return None
    ctx.set_gather_cfg(int(e["shape"]), int(e.get("chunk_pct", 0)))
    return e


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


# ----------------------------------------------------------------------------- pe_redshift

_DL_CACHE = {}


def _dl_grid(zmax, nz):
    key = (float(zmax), int(nz))
    if key not in _DL_CACHE:
        from .cosmology import dl_of_z
        z = np.linspace(0.02, zmax, int(nz))
        _DL_CACHE[key] = (z, dl_of_z(z))
    return _DL_CACHE[key]


def _node_y(store, u, ymin):
    """y = sqrt(a), a = s/u, of each (node, template) pair the store covers, and row n_node the boundary
    point (exmarg/search/pe.py:58-84; 0 where a template has no point)"""
    s = np.asarray(store.s, float)
    nn = s.size
    y = np.zeros((nn + 1, u.size))
    for k in range(nn):
        alo = min(store.alpha_lo[k], ymin * ymin)
        a = s[k] / u
        o = (np.sqrt(a) >= ymin) & (a > alo) & (a < store.alpha_hi[k])
        y[k] = np.where(o, np.sqrt(a), 0.0)
        s_prev = s[k - 1] if k > 0 else 0.0
        low = o & (s_prev / u <= alo)
        y[nn][low] = np.sqrt(float(alo) * (1.0 + 1e-9))
    return y


def pe_redshift(segments, bank, store, rows=None, chunk=8, zmax=8.0, nz=1600, m1_range=(3.0, 150.0), nm1=1600,
                ymin=0.1267, nodes_per_launch=6, block=256, mdet_range=(10.0, 500.0), resident=False, n_loud=1024,
                n_random=1024, seed=0):
    """ln Lambda(m1_source, z) of each segment (the contract of exmarg/search/pe.py:203-257).

    bank: an ascending equal-mass, zero-spin bank of detector-frame total masses.  With a 'b200' bank
    every segment runs filter, time selection and the plane gather on the device (exm_filter,
    exm_select_times, exm_node_values), then the source frame and ln B (exm_source_frame); chunk,
    nodes_per_launch, block and resident are accepted and have no effect.  D_L(z) is
    exmarg_b200.cosmology's restatement of Planck 2018 (the reference uses astropy's Planck18).

    returns dict: m1 (nm1,), z (nz,), ln_lambda (n_segment, nm1, nz), ln_b (n_segment,), rows."""
    if getattr(bank, "device", None) in ("cpu", "gpu"):
        import exmarg.search as ref
        return ref.pe_redshift(segments, bank, store, rows=rows, chunk=chunk, zmax=zmax, nz=nz, m1_range=m1_range,
                               nm1=nm1, ymin=ymin, nodes_per_launch=nodes_per_launch, block=block,
                               mdet_range=mdet_range, resident=resident, n_loud=n_loud, n_random=n_random, seed=seed)
    if getattr(bank, "device", None) != "b200":
        raise ValueError("device must be 'cpu', 'gpu' or 'b200'")
    M = np.asarray(bank.M, float)
    if np.any(np.diff(M) <= 0) or np.any(np.asarray(bank.q) != 1.0) or np.any(np.asarray(bank.chi) != 0.0):
        raise ValueError("pe_redshift needs an ascending equal-mass zero-spin bank")
    from .segments import D0
    seg = read_segments(segments, rows)
    z, dl = _dl_grid(zmax, nz)
    m1 = np.geomspace(m1_range[0], m1_range[1], int(nm1))
    ctx = prepare(bank, store, "volume", ymin)
    key = (ctx.bank_token, ctx.store_token, float(ymin), float(zmax), int(nz), float(m1_range[0]),
           float(m1_range[1]), int(nm1), float(mdet_range[0]), float(mdet_range[1]))
    if getattr(ctx, "rs_key", None) != key:
        lnp = np.log(np.maximum((1.0 + z) * dl ** 2 * np.gradient(dl, z), 1e-300))
        Md = 2.0 * m1[:, None] * (1.0 + z[None, :])
        inside = (Md >= mdet_range[0]) & (Md <= mdet_range[1])
        w = np.where(inside, np.exp(lnp)[None, :], 0.0) * np.gradient(m1)[:, None] * np.gradient(z)[None, :]
        w /= w.sum()
        ctx.redshift_grid(_node_y(store, np.asarray(bank.u, float), ymin), M, D0 / dl, z, m1, w)
        ctx.rs_key = key
    nn = len(store.s)
    out = np.full((seg["rows"].size, m1.size, z.size), -np.inf)
    ln_b = np.empty(seg["rows"].size)
    for e, row in enumerate(seg["rows"]):
        ctx.filter(seg["d_H"][e:e + 1], seg["d_L"][e:e + 1], seg["sig2_H"], seg["sig2_L"], want=False)
        if n_loud > 0:
            ctx.select_times(seed + int(row), n_loud, n_random, want=False)
        else:
            ctx.set_times(None)
        lamN = ctx.node_values(nn)
        out[e], ln_b[e] = ctx.source_frame(lamN)
    return dict(m1=m1, z=z, ln_lambda=out, ln_b=ln_b, rows=seg["rows"])
