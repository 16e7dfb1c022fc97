"""The template bank of the 'b200' device (exmarg/search/bank.py:35-54, MassBank.__init__) against the
reference's own banks: every golden fixture holds the W and u the reference's mass_bank built for its
bank rows and segments (tests/golden/make_golden.py), and exmarg_b200.mass_bank must rebuild them
bit for bit from the same rows (no GPU needed: W and u are formed on the host)."""

import os

import numpy as np
import pytest

from exmarg_b200.bank import MassBank, mass_bank
from tests.golden_io import GOLDEN

CASES = ["config1", "prodshape", "alltimes_md", "redshift1"]


def _segment(z):
    return dict(d_H=z["d_H"], d_L=z["d_L"], f=z["f"], nu=z["nu"], sig2=z["sig2"], T=float(z["T"]),
                fmin=float(z["fmin"]), fmax=float(z["fmax"]))


@pytest.mark.parametrize("name", CASES)
def test_mass_bank_rebuilds_reference_W_and_u(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    bank = mass_bank(z["bank_rows"], _segment(z), device="b200")
    assert bank.W.dtype == np.complex64 and bank.W.shape == z["W"].shape
    assert np.array_equal(bank.W, z["W"])
    assert np.array_equal(bank.u, z["u"])
    assert bank.lo == int(z["lo"]) and bank.n_time == int(z["n_time"])


def test_mass_bank_rejects_gapped_bins():
    z = np.load(os.path.join(GOLDEN, "config1.npz"))
    seg = _segment(z)
    seg["nu"] = np.concatenate([seg["nu"][:5], seg["nu"][6:]])
    rows = z["bank_rows"]
    with pytest.raises(ValueError, match="contiguous"):
        MassBank(rows[:, 0], rows[:, 1], rows[:, 2], dict(seg, sig2_H=z["sig2"]), "b200")
