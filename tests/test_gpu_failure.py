"""Failure detection on the device without a GPU fault: the plane gather's barrier waits are bounded,
and when one runs out the kernel sets the device error word and returns.  The test makes a wait run out
by letting the gather issue no table copy (a barrier that nothing completes, so no copy is ever in flight
when a block exits), checks that the call reports the timeout as a status, and that the same context then
analyses the segment normally."""

import numpy as np
import pytest

import exmarg_b200 as eb
from tests.golden_io import Fixture

pytestmark = pytest.mark.gpu


def test_expired_wait_is_reported_and_context_recovers():
    fx = Fixture("config1")
    bank = fx.b200_bank()
    ctx = eb.prepare(bank, fx.store, fx.prior_arg, fx.ymin)
    kw = dict(prior=fx.prior_arg, ymin=fx.ymin, n_loud=fx.n_loud, n_random=fx.n_random, seed=0)
    ctx.test_wait_expiry(True)
    try:
        with pytest.raises(RuntimeError, match="bounded device wait"):
            eb.pe_intrinsic(fx.seg, bank, fx.store, **kw)
    finally:
        ctx.test_wait_expiry(False)
    res = eb.pe_intrinsic(fx.seg, bank, fx.store, **kw)
    assert np.abs(res["ln_b"] - fx.ln_b).max() <= 1e-5
