"""Stage 1 of the table build on the CPU: the HEALPix RING pixel centres satisfy the scheme's closed
forms, and the oracle's restatement of w_gpu.py's quadrature reproduces the reference's own GORFs
(tests/golden/w1.npz, made by running w_table_s_gpu with numpy standing in for cupy)."""

import os

import numpy as np

from exmarg_b200 import wtable
from oracle import restate

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "w1.npz")


def test_pix2ang_ring_scheme():
    th, ph = wtable.pix2ang(1, np.arange(12))
    z = np.cos(th)
    assert np.allclose(z, np.repeat([2 / 3, 0.0, -2 / 3], 4))
    assert np.allclose(ph, np.array([1, 3, 5, 7, 0, 2, 4, 6, 1, 3, 5, 7]) * np.pi / 4)
    for nside in (2, 4, 8, 32):
        npix = wtable.nside2npix(nside)
        th, ph = wtable.pix2ang(nside, np.arange(npix))
        z = np.cos(th)
        assert np.all(np.diff(z) <= 1e-12)                        # rings from north to south
        assert np.allclose(np.sort(z), -np.sort(z)[::-1])           # symmetric about the equator
        rings, counts = np.unique(np.round(z, 12), return_counts=True)
        assert rings.size == 4 * nside - 1 and counts.sum() == npix
        assert counts.max() == 4 * nside and counts.min() == 4
        assert np.all((ph >= 0) & (ph < 2 * np.pi))
        assert abs(z.mean()) < 1e-12 and abs(np.mean(z ** 2) - 1 / 3) < 0.05 / nside ** 2   # equal area


def test_oracle_matches_reference_w():
    z = np.load(GOLDEN)
    tau, W = restate.w_table_s(z["s"], int(z["n_max"]), int(z["nside"]), int(z["n_tau"]), wtable.pix2ang)
    assert np.allclose(tau, z["tau"], rtol=0, atol=1e-18)
    ref = z["W"]
    scale = np.abs(ref).max(axis=1, keepdims=True)                   # per node and key, over tau
    assert np.all(np.abs(W - ref) <= 1e-12 * scale + 1e-300)
