"""Node shards on the device.  One GPU stands in for the ranks by computing each node range's rows in
turn (no process group: the exchange is the elementwise max that the all-reduce computes).  Each
shard's rows equal the whole store's rows at its nodes, and its boundary row holds exactly the
templates whose boundary node it owns; combined, they give the reference's ln Lambda and ln B.  A
shard context refuses the fused pe_intrinsic (its node log-sum-exp needs every shard)."""

import numpy as np
import pytest

import exmarg_b200 as eb
from exmarg_b200 import shard
from exmarg_b200.pe import prepare
from tests.golden_io import Fixture

pytestmark = pytest.mark.gpu

TOL_ROWS = 1e-12        # node values: the same tables and taps, partial sums in another order at most


def _whole_rows(fx, bank):
    ctx = prepare(bank, fx.store, fx.prior_arg, fx.ymin)
    seg = eb.read_segments(fx.seg)
    out = []
    for e, row in enumerate(seg["rows"]):
        ctx.filter(seg["d_H"][e:e + 1], seg["d_L"][e:e + 1], seg["sig2_H"], seg["sig2_L"], want=False)
        if fx.n_loud > 0:
            ctx.select_times(int(row), fx.n_loud, fx.n_random, want=False)
        else:
            ctx.set_times(None)
        out.append(ctx.node_values(len(fx.store.s)))
    return seg, np.stack(out)


@pytest.mark.parametrize("case", ["config1", "prodshape", "alltimes_md"])
def test_shards_give_the_whole_store_rows(case):
    fx = Fixture(case)
    bank = fx.b200_bank()
    seg, whole = _whole_rows(fx, bank)
    nn = len(fx.store.s)
    _, _, bnode = shard.node_geometry(fx.store.s, fx.store.alpha_lo, fx.store.alpha_hi, fx.u, fx.ymin)
    lnW = shard.node_weights(fx.store, fx.u, fx.ymin, fx.prior_arg)
    for n in range(2, nn + 1):
        ranges = shard.node_ranges(fx.store, fx.u, fx.ymin, n)
        lamN = np.full_like(whole, -np.inf)
        for k0, k1 in ranges:
            part = shard._device_node_values(seg, bank, fx.store, k0, k1, fx.prior_arg, fx.ymin, fx.n_loud,
                                             fx.n_random, 0)
            mine = (bnode >= k0) & (bnode < k1)
            assert np.all(np.isneginf(part[:, k1 - k0, ~mine]))     # boundary points of other ranges: none
            lamN = np.maximum(lamN, shard.place(part, k0, k1, nn))
        assert np.array_equal(np.isfinite(lamN), np.isfinite(whole))
        fin = np.isfinite(whole)
        assert np.abs(lamN[fin] - whole[fin]).max() <= TOL_ROWS * max(1.0, np.abs(whole[fin]).max())
        ln_lambda, ln_b = shard.combine(lamN, lnW, bank.M, bank.q, bank.chi)
        assert np.abs(ln_lambda - fx.ln_lambda).max() < 1e-4
        assert np.abs(ln_b - fx.ln_b).max() < 1e-5


def test_one_rank_sharded_equals_pe_intrinsic():
    fx = Fixture("prodshape")
    kw = dict(prior=fx.prior_arg, ymin=fx.ymin, n_loud=fx.n_loud, n_random=fx.n_random)
    a = shard.pe_intrinsic_sharded(fx.seg, fx.b200_bank(), fx.store, **kw)
    b = eb.pe_intrinsic(fx.seg, fx.b200_bank(), fx.store, **kw)
    assert np.abs(a["ln_lambda"] - b["ln_lambda"]).max() < 1e-12
    assert np.abs(a["ln_b"] - b["ln_b"]).max() < 1e-12


def test_shard_context_refuses_pe_intrinsic():
    fx = Fixture("config1")
    bank = fx.b200_bank()
    sub = shard.shard_of(fx.store, 1, len(fx.store.s))
    prepare(bank, sub, fx.prior_arg, fx.ymin)
    with pytest.raises(RuntimeError, match="shard"):
        eb.pe_intrinsic(fx.seg, bank, sub, prior=fx.prior_arg, ymin=fx.ymin, n_loud=fx.n_loud, n_random=fx.n_random)
