"""Stage 3 of the table build: the oracle's restatement of build_bd.py's log-sum over the orders
reproduces the reference's own tables (tests/golden/bd1.npz, made by running build_bd.build_node on a
synthetic stage-2 store), and the host helpers give the reference's grids and lnK edges."""

import os

import numpy as np

from exmarg_b200 import tables
from oracle import restate

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "bd1.npz")


def test_grid_and_edges():
    z = np.load(GOLDEN)
    beta, delta = tables.bd_grid(z["lnq"])
    assert np.array_equal(beta, z["beta"]) and np.array_equal(delta, z["delta"])
    col, row = tables.lnk_edges(z["lnK"])
    assert np.array_equal(col, z["lnK"][:, :, :, -1, :col.shape[3]])
    assert np.array_equal(row, z["lnK"][:, :, -1, :, :col.shape[3]])


def test_oracle_matches_reference_tables():
    z = np.load(GOLDEN)
    col, row = tables.lnk_edges(z["lnK"])
    ladder = [int(v) for v in z["ladder"]]
    got = restate.bd_tables(col, row, z["lnq"], z["beta"], ladder)
    for nm in ladder:
        ref = z["T%d" % nm]
        assert got[nm].dtype == np.float32 and got[nm].shape == ref.shape
        assert np.array_equal(got[nm], ref), (nm, int(np.sum(got[nm] != ref)))
