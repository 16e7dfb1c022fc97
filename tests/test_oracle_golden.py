"""The oracle (CPU restatement, oracle/) pinned against the reference's own outputs.

The golden vectors were produced by running the reference's CPU path
(exmarg.search, numpy + numba) on seeded inputs (tests/golden/make_golden.py)."""

import numpy as np
import pytest

from oracle import restate
from tests.golden_io import Fixture

CASES = ["config1", "prodshape", "alltimes_md"]


@pytest.fixture(scope="module", params=CASES)
def fx(request):
    return Fixture(request.param)


def test_fixture_tables_regenerate(fx):
    # the float32 generator is deterministic: two regenerations are identical
    T0 = fx.store.tables[0]
    assert T0.dtype == np.float32 and T0.shape == fx.spec.shape
    assert np.isfinite(T0).all()


def test_oracle_pe_intrinsic_matches_reference(fx):
    seg = restate.read_segments(fx.seg)
    M, q, chi = (fx.rows[:, i] for i in range(3))
    res = restate.pe_intrinsic(seg, fx.W, fx.u, M, q, chi, fx.lo, fx.n_time, fx.store, prior=fx.prior, ymin=fx.ymin,
                               n_loud=fx.n_loud, n_random=fx.n_random, seed=0, precision="ref", density=fx.density)
    assert np.allclose(res["ln_lambda"], fx.ln_lambda, rtol=0, atol=1e-9)
    assert np.allclose(res["ln_b"], fx.ln_b, rtol=0, atol=1e-9)


def test_oracle_select_times_matches_reference(fx):
    if "sel0" not in fx.z:
        pytest.skip("every arrival time is walked in this case")
    seg = restate.read_segments(fx.seg)
    traj = restate.trajectories(fx.W, {I: seg["d_" + I][0] for I in "HL"}, {I: seg["sig2_" + I] for I in "HL"},
                                fx.lo, fx.n_time, "ref")
    sel, lw = restate.select_times(traj, fx.store.tau_idx, fx.n_loud, fx.n_random, 0)
    assert np.array_equal(sel, fx.z["sel0"])
    assert np.array_equal(lw, fx.z["lw0"])


def test_oracle_gather_matches_reference(fx):
    seg = restate.read_segments(fx.seg)
    traj = restate.trajectories(fx.W, {I: seg["d_" + I][0] for I in "HL"}, {I: seg["sig2_" + I] for I in "HL"},
                                fx.lo, fx.n_time, "ref")
    times = (fx.z["sel0"], fx.z["lw0"]) if "sel0" in fx.z else None
    tab = fx.z["gather_tab"]
    out = restate.gather(traj, fx.store.tables[:tab.shape[1]], np.arange(fx.u.size), fx.z["gather_lna"], tab,
                         fx.spec.beta, fx.spec.delta, fx.spec.tau_idx, times)
    assert np.allclose(out, fx.z["gather_out"], rtol=0, atol=1e-10)


def test_fp64_oracle_close_to_reference(fx):
    # the all-float64 oracle differs from the reference only by its complex64 filter rounding
    seg = restate.read_segments(fx.seg)
    M, q, chi = (fx.rows[:, i] for i in range(3))
    res = restate.pe_intrinsic(seg, fx.W, fx.u, M, q, chi, fx.lo, fx.n_time, fx.store, prior=fx.prior, ymin=fx.ymin,
                               n_loud=fx.n_loud, n_random=fx.n_random, seed=0, precision="fp64", density=fx.density)
    assert np.abs(res["ln_b"] - fx.ln_b).max() < 1e-4
