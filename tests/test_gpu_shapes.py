"""Every launch shape and template-chunk size of the plane gather gives the reference's results
(the shape changes only the order of the float32 merges), and the autotuner keeps a valid choice."""

import numpy as np
import pytest

import exmarg_b200 as eb
from exmarg_b200 import _lib
from tests.golden_io import Fixture

pytestmark = pytest.mark.gpu

TOL_LNB = 1e-5


def _pe(fx, bank):
    return eb.pe_intrinsic(fx.seg, bank, fx.store, prior=fx.prior_arg, ymin=fx.ymin, n_loud=fx.n_loud,
                           n_random=fx.n_random, seed=0)


@pytest.mark.parametrize("name", ["config1", "prodshape"])
def test_every_shape_and_chunk_matches_reference(name):
    fx = Fixture(name)
    bank = fx.b200_bank()
    ctx = eb.prepare(bank, fx.store, fx.prior_arg, fx.ymin)
    try:
        for cfg in range(len(_lib.GATHER_SHAPES)):
            for pct in (100, 50, 200):
                ctx.set_gather_cfg(cfg, pct)
                res = _pe(fx, bank)
                err = np.abs(res["ln_b"] - fx.ln_b).max()
                assert err <= TOL_LNB, (_lib.GATHER_SHAPES[cfg], pct, err)
                assert np.abs(res["ln_lambda"] - fx.ln_lambda).max() <= 1e-4
    finally:
        ctx.set_gather_cfg(0, 150)


def test_autotune_keeps_a_valid_choice():
    fx = Fixture("config1")
    bank = fx.b200_bank()
    try:
        best, ms = eb.autotune(bank, fx.store, fx.seg, prior=fx.prior_arg, ymin=fx.ymin, n_loud=fx.n_loud,
                               n_random=fx.n_random, reps=1)
        ns = len(_lib.GATHER_SHAPES)
        assert 0 <= best < ns
        assert np.all(ms[:ns + 3] > 0)
        assert bank.ctx.gather_chunk_pct in (50, 100, 150, 200)
        res = _pe(fx, bank)
        assert np.abs(res["ln_b"] - fx.ln_b).max() <= TOL_LNB
    finally:
        bank.ctx.set_gather_cfg(0, 150)


def test_bad_shape_is_rejected():
    fx = Fixture("config1")
    ctx = eb.prepare(fx.b200_bank(), fx.store, fx.prior_arg, fx.ymin)
    with pytest.raises(ValueError):
        ctx.set_gather_cfg(len(_lib.GATHER_SHAPES), 100)
    with pytest.raises(ValueError):
        ctx.set_gather_cfg(0, 5)


def test_autotune_cache_reaches_a_new_context(tmp_path, monkeypatch):
    """autotune(cache=True) records the choice; a fresh context of the same workload takes it without tuning"""
    monkeypatch.setenv("EXMARG_B200_TUNE_CACHE", str(tmp_path / "autotune.json"))
    fx = Fixture("config1")
    kw = dict(prior=fx.prior_arg, ymin=fx.ymin, n_loud=fx.n_loud, n_random=fx.n_random)
    a, b = _lib.Context(0), _lib.Context(0)
    try:
        bank_a = fx.b200_bank()
        bank_a._ctx = a
        best, _ = eb.autotune(bank_a, fx.store, fx.seg, reps=1, **kw)
        bank_b = fx.b200_bank()
        bank_b._ctx = b
        res = eb.pe_intrinsic(fx.seg, bank_b, fx.store, **kw)
        assert b.gather_cfg == best and b.gather_chunk_pct == a.gather_chunk_pct
        assert np.abs(res["ln_b"] - fx.ln_b).max() <= 1e-5
    finally:
        a.close()
        b.close()
