"""Stage 2 of the table build on the CPU: the host restatement of build_k.py's node loading (the delay
rebin onto the data grid) reproduces the reference's W bit for bit, and the oracle's lnK edges reproduce
the reference's lnK (tests/golden/k1.npz: the reference's own load_node, compile_order and build_bd on the
reference's stage-1 output for one node)."""

import os
import tempfile

import numpy as np

from exmarg_b200 import tables, wtable
from oracle import restate

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "k1.npz")


def _stem(z, d):
    stem = os.path.join(d, "sladder_n%03d_s%09.3f" % (int(z["n_max"]), float(z["s"])))
    wtable.save_node(stem, float(z["s"]), z["W_tau"], z["W"], int(z["n_max"]), 2)
    return stem


def test_load_w_node_matches_reference():
    z = np.load(GOLDEN)
    with tempfile.TemporaryDirectory() as d:
        keys, Wd, tau_idx, s, n_max = tables.load_w_node(_stem(z, d))
    assert np.array_equal(keys, z["keys"]) and np.array_equal(tau_idx, z["tau_idx"])
    assert np.array_equal(Wd, z["WM"]) and s == float(z["s"]) and n_max == int(z["n_max"])


def test_oracle_edges_match_reference():
    z = np.load(GOLDEN)
    nphi = int(z["nphi"])
    col, row = restate.k_edges(z["keys"], z["WM"], float(z["s"]), int(z["n_max"]), z["lnq"], nphi)
    nphif = nphi // 2 + 1
    ref_col = z["lnK"][:, :, :, -1, :nphif]
    ref_row = z["lnK"][:, :, -1, :, :nphif]
    assert np.array_equal(col, ref_col) and np.array_equal(row, ref_row)
