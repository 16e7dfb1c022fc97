"""Serving and graph replay: a request's results do not depend on how it was run (bitwise equal
to the plain pe_intrinsic call), and child contexts share the store safely."""

import numpy as np
import pytest

import exmarg_b200 as eb
from exmarg_b200 import MassBank, _lib, synth
from exmarg_b200.serve import Request, Server, latency_stats
from exmarg_b200.store import upload_store
from tests.golden_io import Fixture

pytestmark = pytest.mark.gpu


def _sub_bank(fx, idx):
    M, q, chi = (fx.rows[idx, i] for i in range(3))
    return MassBank(M, q, chi, fx.seg, "b200", W=fx.W[idx], u=fx.u[idx])


def _pe(fx, bank, rows=None):
    return eb.pe_intrinsic(fx.seg, bank, fx.store, rows=rows, prior=fx.prior_arg, ymin=fx.ymin, n_loud=fx.n_loud,
                           n_random=fx.n_random, seed=0)


@pytest.mark.parametrize("name", ["config1", "prodshape", "alltimes_md"])
def test_graph_replay_matches_plain(name):
    fx = Fixture(name)
    bank = fx.b200_bank()
    plain = _pe(fx, bank)
    ctx = bank.ctx
    ctx.set_graph(True)
    try:
        first = _pe(fx, bank)        # segment 0 runs and is captured, segment 1 replays
        again = _pe(fx, bank)        # replays both
    finally:
        ctx.set_graph(False)
    for r in (first, again):
        assert np.array_equal(r["ln_lambda"], plain["ln_lambda"])
        assert np.array_equal(r["ln_b"], plain["ln_b"])


def _mix(fx, keys, n):
    rng = np.random.default_rng(5)
    return [(keys[rng.integers(len(keys))], int(rng.integers(fx.seg["d_H"].shape[0]))) for _ in range(n)]


@pytest.mark.parametrize("budget", ["ample", "one_worker"])
def test_served_results_equal_plain(budget):
    fx = Fixture("config1")
    # a bank on segments of half the duration (half n_time) beside the fixture's: same store and lags
    short_seg = synth.make_segments(2, 321, T=fx.seg["T"] / 2, fmin=fx.seg["fmin"], fmax=fx.seg["fmax"], snr=12.0)
    short = MassBank(fx.rows[:, 0], fx.rows[:, 1], fx.rows[:, 2], short_seg, "b200")
    banks = {"all": fx.b200_bank(), "odd": _sub_bank(fx, np.arange(1, 64, 2)), "low": _sub_bank(fx, np.arange(20)),
             "short": short}
    segs = {k: fx.seg for k in banks}
    segs["short"] = short_seg
    expect = {}
    for k, b in banks.items():
        r = eb.pe_intrinsic(segs[k], b, fx.store, prior=fx.prior_arg, ymin=fx.ymin, n_loud=fx.n_loud,
                            n_random=fx.n_random, seed=0)
        for row in range(segs[k]["d_H"].shape[0]):
            expect[(k, row)] = (r["ln_lambda"][row], float(r["ln_b"][row]))
    mix = _mix(fx, sorted(banks), 16)
    reqs = [Request(i, k, segs[k], row=row, seed=0) for i, (k, row) in enumerate(mix)]
    srv = Server(fx.store, banks, max_workers=3, prior=fx.prior_arg, ymin=fx.ymin, n_loud=fx.n_loud,
                 n_random=fx.n_random)
    if budget == "one_worker":     # one worker at a time: banks take turns, idle ones are evicted
        srv.sched.max_workers = 1
    try:
        done = srv.serve(reqs, arrivals=np.linspace(0.0, 0.05, len(reqs)))
        peak_workers = srv.sched.n_workers()
        assert srv.sched.used <= srv.sched.budget
    finally:
        srv.close()
    for r in done:
        lnl, lnb = r.future.result()
        e_lnl, e_lnb = expect[(r.key, r.row)]
        assert np.array_equal(lnl, e_lnl) and lnb == e_lnb
    st = latency_stats(done)
    assert st["requests"] == len(reqs) and st["p99_ms"] >= st["p50_ms"] > 0
    if budget == "one_worker":
        assert peak_workers == 1


def test_child_context_borrows_store():
    fx = Fixture("config1")
    parent = _lib.Context(0)
    upload_store(fx.store, parent)
    child = _lib.Context(share_store_of=parent)
    bank = fx.b200_bank().clone_for(child)
    try:
        with pytest.raises(RuntimeError, match="child contexts borrow this store"):
            parent.store_init(1, fx.spec.shape, fx.spec.tau_idx, 0.0, 1.0, 0.0, 1.0)
        parent.close()               # deferred: the child still reads the tables
        res = eb.pe_intrinsic(fx.seg, bank, fx.store, prior=fx.prior_arg, ymin=fx.ymin, n_loud=fx.n_loud,
                              n_random=fx.n_random, seed=0)
        assert np.abs(res["ln_b"] - fx.ln_b).max() <= 1e-5
    finally:
        child.close()                # frees the parent's tables too
