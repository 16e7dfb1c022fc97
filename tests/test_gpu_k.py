"""Stage 2 on the device (exm_k_edges) and the fused stage 2 + 3 (build_node_from_w), against the
reference's own lnK and tables (tests/golden/k1.npz) and the oracle.

Bars: lnK edges within 2 float32 ulp of the reference where K_n stands clear of cancellation (the log part
above -500); where the reference's K_n cancelled to its 1e-300 floor (log part below -600: rounding noise
of sums whose terms are ~1e-16 of the largest), the device's is below -500 too (both are nothing next to the
other orders in stage 3).  Tables within 2 ulp of the reference's."""

import os

import numpy as np
import pytest

from exmarg_b200 import _lib, tables, wtable
from oracle import restate

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "k1.npz")


def ulps(a, b):
    ia = a.view(np.int32).astype(np.int64)
    ib = b.view(np.int32).astype(np.int64)
    ia = np.where(ia < 0, -(ia & 0x7FFFFFFF), ia)
    ib = np.where(ib < 0, -(ib & 0x7FFFFFFF), ib)
    return np.abs(ia - ib)


def _check_edges(got, ref, gmo):
    lg_ref = ref.astype(np.float64) - gmo[:, None, None, None]
    lg_got = got.astype(np.float64) - gmo[:, None, None, None]
    clear = lg_ref > -500
    assert np.all(ulps(got, ref)[clear] <= 2), int(ulps(got, ref)[clear].max())
    floor = lg_ref < -600
    assert np.all(lg_got[floor] < -500)
    return int(clear.sum()), int(floor.sum())


def test_edges_match_reference():
    z = np.load(GOLDEN)
    nphi, n_max = int(z["nphi"]), int(z["n_max"])
    coeff, gmo, cosm = tables.k_inputs(z["keys"], float(z["s"]), n_max, z["lnq"], nphi)
    col, row, _ = _lib.context(0).k_edges(n_max, z["WM"], coeff, z["lnq"], gmo, cosm)
    nphif = nphi // 2 + 1
    _check_edges(col, np.ascontiguousarray(z["lnK"][:, :, :, -1, :nphif]), gmo)
    _check_edges(row, np.ascontiguousarray(z["lnK"][:, :, -1, :, :nphif]), gmo)


def test_fused_build_matches_reference_table(tmp_path):
    z = np.load(GOLDEN)
    stem = os.path.join(str(tmp_path), "sladder_n%03d_s%09.3f" % (int(z["n_max"]), float(z["s"])))
    wtable.save_node(stem, float(z["s"]), z["W_tau"], z["W"], int(z["n_max"]), 2)
    f = tables.build_node_from_w(stem, os.path.join(str(tmp_path), "bd"), nq=z["lnq"].size, nphi=int(z["nphi"]))
    out = np.load(f[0])
    assert np.array_equal(out["beta"], z["beta"]) and np.array_equal(out["delta"], z["delta"])
    assert np.array_equal(out["tau_idx"], z["tau_idx"])
    d = ulps(out["T"], z["T"])
    assert d.max() <= 2, (int(d.max()), int((d > 0).sum()))


def test_edges_against_oracle_more_orders():
    """12 orders (several phase classes of up to 12 rows, two row chunks of the class kernel) on
    synthetic W with the production magnitude grid"""
    rng = np.random.default_rng(3)
    n_max, n_tau, nphi = 11, 9, 96
    keys = np.array(wtable.keys(n_max))
    Wd = np.exp(rng.normal(-3.0, 1.0, (keys.shape[0], n_tau))) * (1 + 0.1 * rng.standard_normal((keys.shape[0], 1)))
    lnq = np.log(np.geomspace(0.05, 100.0, 110))
    s = 2.5
    coeff, gmo, cosm = tables.k_inputs(keys, s, n_max, lnq, nphi)
    col, row, _ = _lib.context(0).k_edges(n_max, Wd, coeff, lnq, gmo, cosm)
    rc, rr = restate.k_edges(keys, Wd, s, n_max, lnq, nphi)
    _check_edges(col, rc, gmo)
    _check_edges(row, rr, gmo)


def test_cli_from_w(tmp_path):
    """python -m exmarg_b200.tables from-w on the golden node; a second run finds the table and skips it"""
    z = np.load(GOLDEN)
    w_dir = os.path.join(str(tmp_path), "w")
    os.makedirs(w_dir)
    stem = os.path.join(w_dir, "sladder_n%03d_s%09.3f" % (int(z["n_max"]), float(z["s"])))
    wtable.save_node(stem, float(z["s"]), z["W_tau"], z["W"], int(z["n_max"]), 2)
    out = os.path.join(str(tmp_path), "bd")
    assert tables.main(["from-w", w_dir, out, "--nq", str(z["lnq"].size), "--nphi", str(int(z["nphi"]))]) == 0
    f = os.path.join(out, "bd_n%03d_s%09.3f.npz" % (int(z["n_max"]), float(z["s"])))
    assert ulps(np.load(f)["T"], z["T"]).max() <= 2
    assert tables.build_node_from_w(stem, out, nq=z["lnq"].size, nphi=int(z["nphi"])) == []
