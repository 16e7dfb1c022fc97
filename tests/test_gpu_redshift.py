"""pe_redshift on the B200 (filter, selection and plane gather on the device, then the source frame
and ln B in exm_source_frame) against the reference's outputs (tests/golden/redshift1.npz), and the
device source frame alone against the oracle's restatement on the same node values."""

import numpy as np
import pytest

import exmarg_b200 as eb
from exmarg_b200 import MassBank
from exmarg_b200.pe import _dl_grid, _node_y
from oracle import restate
from tests.test_oracle_redshift import load

pytestmark = pytest.mark.gpu


def _bank(z, seg):
    r = z["bank_rows"]
    return MassBank(r[:, 0], r[:, 1], r[:, 2], seg, "b200", W=z["W"], u=z["u"])


def _run(z, store, seg, bank):
    return eb.pe_redshift(seg, bank, store, zmax=float(z["zmax"]), nz=int(z["nz"]),
                          m1_range=(float(z["m1_lo"]), float(z["m1_hi"])), nm1=int(z["nm1"]), n_loud=int(z["n_loud"]),
                          n_random=int(z["n_random"]), seed=0)


def test_pe_redshift_matches_reference():
    z, spec, store, seg = load()
    res = _run(z, store, seg, _bank(z, seg))
    ref = z["ln_lambda"]
    assert np.array_equal(res["z"], z["z"]) and np.array_equal(res["m1"], z["m1"])
    fin = np.isfinite(ref)
    # the surface interpolates the node values: the gather's float32 tables give the same bar as pe_intrinsic
    assert np.array_equal(np.isfinite(res["ln_lambda"]), fin)
    assert np.abs(res["ln_lambda"][fin] - ref[fin]).max() <= 1e-4
    assert np.abs(res["ln_b"] - z["ln_b"]).max() <= 1e-5


def test_source_frame_equals_restatement_on_same_node_values():
    z, spec, store, seg = load()
    bank = _bank(z, seg)
    res = _run(z, store, seg, bank)            # sets the grid on the bank's context
    ctx = bank.ctx
    rng = np.random.default_rng(4)
    nn1, nm = len(store.s) + 1, z["u"].size
    yN = _node_y(store, z["u"], 0.1267)
    lamN = np.where(yN > 0, rng.normal(20.0, 8.0, (nn1, nm)), -np.inf)
    lamN[:, 3] = -np.inf                          # a template with no point at all
    out, lnb = ctx.source_frame(lamN)
    zz, dl = _dl_grid(float(z["zmax"]), int(z["nz"]))
    ref = restate.source_frame(lamN, yN, z["bank_rows"][:, 0], eb.D0 / dl, res["m1"], zz)
    assert np.array_equal(np.isfinite(out), np.isfinite(ref))
    fin = np.isfinite(ref)
    assert np.array_equal(out[fin], ref[fin])      # the same float64 operations in the same order
    w = restate.redshift_weights(res["m1"], zz, dl, (10.0, 500.0))
    assert abs(lnb - restate.log_mean(ref, w)) <= 1e-12


def test_pe_redshift_rejects_unequal_mass_bank():
    z, spec, store, seg = load()
    r = z["bank_rows"].copy()
    r[:, 1] = 0.8
    bank = MassBank(r[:, 0], r[:, 1], r[:, 2], seg, "b200", W=z["W"], u=z["u"])
    with pytest.raises(ValueError):
        eb.pe_redshift(seg, bank, store, nz=10, nm1=10)
