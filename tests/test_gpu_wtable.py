"""Stage 1 of the table build on the device (exm_w_build): the reference's own GORFs (golden w1), the
oracle at n_max 20 (several tiles per phase class, partial tiles on both axes), at 53 nodes (the
production node count) and at 64 (every row of a tile), build_w's files, and the refusal of a delay bin outside the grid.

Bars, relative to the largest |W| of each (node, key) over tau, beyond two float32 subnormal steps
(at s = 0.01 the high orders are near 1e-40, where float32 keeps only a few bits, as the reference's
float32 tables do):
* against the oracle with |R| and arg R rounded to float32 from float64, as the device forms them:
  1e-7 (the float32 result, float64 sums taken in another order);
* against the reference's golden W: 1e-6.  The reference forms the detector responses in float32, and
  the float32 |R| and arg R of numpy (which made the golden), of CUDA (the reference's cupy run) and of a
  correctly rounded evaluation differ in the last bit; through the damping exp(-s |R|^2) that moves W by
  up to 3.3e-7 of its scale at s = 20 (the oracle rounded like the device is 3.31e-7 from the golden too)."""

import os

import numpy as np
import pytest

from exmarg_b200 import _lib, wtable
from oracle import restate

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "w1.npz")
TOL = 1e-7
TOL_REF = 1e-6


SUB = 2.0 ** -149     # float32's subnormal spacing: W below 1.2e-38 (small s, high order) keeps fewer bits


def _close(W, ref):
    """the largest |W - ref| over the bar's unit (the largest |ref| of the (node, key) over tau), after
    allowing two subnormal steps of float32"""
    scale = np.abs(ref).max(axis=1, keepdims=True)
    err = np.maximum(np.abs(W.astype(np.float64) - ref) - 2 * SUB, 0.0) / np.maximum(scale, 1e-300)
    return float(err.max())


def test_reference_w():
    z = np.load(GOLDEN)
    tau, W, _ = wtable.w_table(z["s"], int(z["n_max"]), int(z["nside"]), int(z["n_tau"]))
    assert np.allclose(tau, z["tau"], rtol=0, atol=1e-18)
    assert _close(W, z["W"]) < TOL_REF
    _, ref = restate.w_table_s(z["s"], int(z["n_max"]), int(z["nside"]), int(z["n_tau"]), wtable.pix2ang, "correct")
    assert _close(W, ref) < TOL


@pytest.mark.parametrize("s, n_max, nside, n_tau", [
    (np.geomspace(0.01, 200.0, 4), 20, 2, 33),
    (np.geomspace(4.3e-3, 4000.0, 53), 3, 1, 9),      # the production node count
    (np.geomspace(4.3e-3, 4000.0, 64), 3, 1, 9),      # every row of the 64-row tile
])
def test_against_oracle(s, n_max, nside, n_tau):
    tau, W, _ = wtable.w_table(s, n_max, nside, n_tau)
    _, ref = restate.w_table_s(s, n_max, nside, n_tau, wtable.pix2ang, "correct")
    assert W.shape == ref.shape and np.isfinite(W).all()
    assert _close(W, ref) < TOL


def test_build_w_files(tmp_path):
    z = np.load(GOLDEN)
    wtable.build_w(str(tmp_path), z["s"], int(z["n_max"]), int(z["nside"]), int(z["n_tau"]))
    ks = wtable.keys(int(z["n_max"]))
    for j, s in enumerate(z["s"]):
        stem = os.path.join(str(tmp_path), "sladder_n%03d_s%09.3f" % (int(z["n_max"]), s))
        Wf = np.load(stem + ".W.npy")
        meta = np.load(stem + ".meta.npz")
        assert Wf.dtype == np.float32 and Wf.shape == (len(ks), int(z["n_tau"]))
        assert np.array_equal(meta["keys"], np.array(ks, np.int16)) and float(meta["s_node"]) == s
        assert _close(Wf.T[None], z["W"][j:j + 1]) < TOL_REF
    assert int(np.load(os.path.join(str(tmp_path), "manifest.npz"))["n_max"]) == int(z["n_max"])


def test_refuses_bad_delay_bin():
    g = wtable.geometry(1, 2, 9)
    g["j0"] = g["j0"].copy()
    g["j0"][3] = 8                       # the upper bin j0 + 1 would lie outside the 9-point grid
    with pytest.raises(ValueError):
        _lib.context(0).w_build(np.array([1.0]), 2, g, wtable.scales([1.0], 2))
