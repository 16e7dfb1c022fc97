"""Stage 3 of the table build on the device (exm_bd_build): the reference's own tables (golden bd1, every
truncation order of its ladder), a production-shape node (121 orders, 87 lags, 110 magnitudes, 49 phases)
against the oracle on sampled lags, build_node's files end to end, and the refusal of a table with a
non-finite entry.  Bar: float32 results within one unit in the last place of the reference's (the
float64 exp and log of the device and of numpy may differ in their last bit)."""

import os

import numpy as np
import pytest

from exmarg_b200 import _lib, tables
from oracle import restate

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "bd1.npz")


def ulps(a, b):
    ia = a.view(np.int32).astype(np.int64)
    ib = b.view(np.int32).astype(np.int64)
    ia = np.where(ia < 0, -(ia & 0x7FFFFFFF), ia)
    ib = np.where(ib < 0, -(ib & 0x7FFFFFFF), ib)
    return np.abs(ia - ib)


def edges(nord, ntau, nq, nphif, seed):
    """synthetic lnK edges: 2n ln max(q1, q2) plus a function of ln q1 - ln q2, Poisson-like in n"""
    from scipy.special import gammaln
    rng = np.random.default_rng(seed)
    lnq = np.log(np.geomspace(0.05, 100.0, nq))
    n = np.arange(nord, dtype=np.float64)[:, None, None, None]
    t = np.arange(ntau, dtype=np.float64)[None, :, None, None]
    ph = (2 * np.pi * np.arange(nphif) / (2 * (nphif - 1)))[None, None, None, :]
    dq = np.abs(lnq - lnq[-1])[None, None, :, None]
    base = n * (0.4 * np.cos(ph) + 0.01 * t - 0.3 * dq) - gammaln(n + 1.0)
    col = (2 * n * lnq[-1] + base + 0.01 * rng.standard_normal(base.shape)).astype(np.float32)
    row = (2 * n * lnq[None, None, :, None] + base + 0.01 * rng.standard_normal(base.shape)).astype(np.float32)
    return col, row, lnq


def test_reference_tables():
    z = np.load(GOLDEN)
    col, row = tables.lnk_edges(z["lnK"])
    ladder = [int(v) for v in z["ladder"]]
    Ts, beta, delta, _ = tables.bd_tables(col, row, z["lnq"], ladder)
    assert np.array_equal(beta, z["beta"]) and np.array_equal(delta, z["delta"])
    for nm in ladder:
        d = ulps(Ts[nm], z["T%d" % nm])
        assert d.max() <= 1 and np.mean(d > 0) < 1e-3, (nm, int(d.max()), int(np.sum(d > 0)))


def test_production_shape_against_oracle():
    col, row, lnq = edges(121, 87, 110, 49, 5)
    Ts, beta, delta, stats = tables.bd_tables(col, row, lnq)
    T = Ts[120]
    assert T.shape == (87, 49, 200, 219) and np.isfinite(T).all()
    for t in (0, 86):
        ref = restate.bd_tables(col[:, t:t + 1], row[:, t:t + 1], lnq, beta, [120])[120][0]
        d = ulps(T[t], ref)
        assert d.max() <= 1 and np.mean(d > 0) < 1e-3, (t, int(d.max()), int(np.sum(d > 0)))


def test_build_node_files(tmp_path):
    z = np.load(GOLDEN)
    nord = z["lnK"].shape[0]
    stem = os.path.join(str(tmp_path), "kstore_n%03d_s%09.3f" % (nord - 1, float(z["s"])))
    np.save(stem + ".lnK.npy", z["lnK"])
    np.savez(stem + ".meta.npz", s_node=float(z["s"]), lnq=z["lnq"], tau_idx=z["tau_idx"])
    base = os.path.join(str(tmp_path), "bd")
    ladder = [int(v) for v in z["ladder"]]
    files = tables.build_node(stem, base, ladder)
    assert len(files) == len(ladder)
    for nm in ladder:
        f = os.path.join(tables.out_dir(base, nm, nord - 1), "bd_n%03d_s%09.3f.npz" % (nm, float(z["s"])))
        out = np.load(f)
        assert ulps(out["T"], z["T%d" % nm]).max() <= 1
        assert int(out["n_max"]) == nm and int(out["nphif"]) == out["T"].shape[1] and str(out["norm"]) == "taylor_off1"
        assert np.array_equal(out["beta"], z["beta"]) and np.array_equal(out["tau_idx"], z["tau_idx"])
    assert tables.build_node(stem, base, ladder) == []          # written tables are skipped


def test_non_finite_table_refused():
    z = np.load(GOLDEN)
    col, row = tables.lnk_edges(z["lnK"])
    col = col.copy()
    col[3, 1, 4, 2] = np.nan
    with pytest.raises(FloatingPointError):
        tables.bd_tables(col, row, z["lnq"])
    ctx = _lib.context(0)
    with pytest.raises(ValueError):
        ctx.bd_build(col, row, z["lnq"], z["beta"], [col.shape[0]])     # truncation order beyond the orders
