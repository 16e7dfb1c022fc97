"""The native request loop (exm_serve_start / exm_submit / exm_poll), driven through the C ABI only.

A request is one row of pe_intrinsic (exmarg/search/pe.py:289-346) for one of the server's banks; the
loop runs requests of several banks at once on child contexts.  Every served result must be bitwise the
result of exm_pe_intrinsic on the parent context for the same bank, segment and seed."""

import numpy as np
import pytest

import exmarg_b200 as eb
from exmarg_b200 import MassBank, _lib
from tests.golden_io import Fixture

pytestmark = pytest.mark.gpu


def _setup():
    fx = Fixture("config1")
    big = fx.b200_bank()
    ctx = eb.prepare(big, fx.store, fx.prior_arg, fx.ymin)
    ctx.set_gather_cfg(0, 150)
    M, q, chi = (fx.rows[:24, i] for i in range(3))
    small = MassBank(M, q, chi, fx.seg, "b200", W=fx.W[:24], u=fx.u[:24])
    seg = eb.read_segments(fx.seg)
    return fx, ctx, {"big": big, "small": small}, seg


def _plain(fx, banks, seg, mix):
    out = []
    for key, row, seed in mix:
        r = eb.pe_intrinsic(fx.seg, banks[key], fx.store, rows=[row], prior=fx.prior_arg, ymin=fx.ymin,
                            n_loud=fx.n_loud, n_random=fx.n_random, seed=seed)
        out.append((r["ln_lambda"][0], float(r["ln_b"][0])))
    return out


def test_submit_poll_mixed_banks_bitwise_plain():
    fx, ctx, banks, seg = _setup()
    mix = [("big", 0, 0), ("small", 1, 3), ("big", 1, 5), ("small", 0, 0), ("big", 0, 7), ("small", 1, 1),
           ("big", 1, 0), ("small", 0, 9)]
    want = _plain(fx, banks, seg, mix)
    ctx.serve_start(hbm_budget=0, max_workers=2, n_loud=fx.n_loud, n_random=fx.n_random)
    try:
        ids = {k: ctx.serve_add_bank(b.W, b.lo, b.n_time, b.u, b.M, b.q, b.chi, fx.ymin) for k, b in banks.items()}
        handles = []
        for key, row, seed in mix:
            handles.append(ctx.submit(ids[key], seg["d_H"][row], seg["d_L"][row], seg["sig2_H"], seg["sig2_L"],
                                      seed + row))
        first = ctx.poll(handles[0], banks["big"].u.size, timeout_us=0)   # may not have finished yet
        got = [first if first is not None else ctx.poll(handles[0], banks["big"].u.size)]
        for h, (key, _, _) in zip(handles[1:], mix[1:]):
            got.append(ctx.poll(h, banks[key].u.size, timeout_us=-1))
        for (lnl, lnb), (wl, wb) in zip(got, want):
            assert np.array_equal(lnl, wl) and lnb == wb
        st = ctx.serve_stats()
        assert st["served"] == len(mix) and st["failed"] == 0 and st["queued"] == 0 and st["running"] == 0
        assert 1 <= st["workers"] <= 2
        with pytest.raises(ValueError, match="unknown request handle"):
            ctx.poll(handles[0], banks["big"].u.size)            # a handle is released by its result
    finally:
        ctx.serve_stop()


def test_budget_closes_idle_workers_of_other_banks():
    # room for one worker only: requests alternate banks, so each bank change closes the other bank's
    # idle worker and opens one of its own; results stay bitwise the plain path's
    fx, ctx, banks, seg = _setup()
    mix = [("big", 0, 0), ("small", 1, 0), ("big", 1, 0)]
    want = _plain(fx, banks, seg, mix)
    ctx.serve_start(hbm_budget=0, max_workers=1, n_loud=fx.n_loud, n_random=fx.n_random)
    try:
        ids = {k: ctx.serve_add_bank(b.W, b.lo, b.n_time, b.u, b.M, b.q, b.chi, fx.ymin) for k, b in banks.items()}
        for (key, row, seed), (wl, wb) in zip(mix, want):
            h = ctx.submit(ids[key], seg["d_H"][row], seg["d_L"][row], seg["sig2_H"], seg["sig2_L"], seed + row)
            lnl, lnb = ctx.poll(h, banks[key].u.size)
            assert np.array_equal(lnl, wl) and lnb == wb
        st = ctx.serve_stats()
        assert st["workers_opened"] == 3 and st["workers_closed"] == 2 and st["workers"] == 1
    finally:
        ctx.serve_stop()


def test_serve_errors():
    fx, ctx, banks, seg = _setup()
    with pytest.raises(RuntimeError, match="no server"):
        ctx.submit(0, seg["d_H"][0], seg["d_L"][0], seg["sig2_H"], seg["sig2_L"], 0)
    ctx.serve_start(max_workers=1, n_loud=fx.n_loud, n_random=fx.n_random)
    try:
        with pytest.raises(RuntimeError, match="already running"):
            ctx.serve_start()
        b = banks["small"]
        bid = ctx.serve_add_bank(b.W, b.lo, b.n_time, b.u, b.M, b.q, b.chi, fx.ymin)
        with pytest.raises(ValueError, match="unknown bank"):
            ctx.submit(bid + 1, seg["d_H"][0], seg["d_L"][0], seg["sig2_H"], seg["sig2_L"], 0)
        h = ctx.submit(bid, seg["d_H"][0], seg["d_L"][0], seg["sig2_H"], seg["sig2_L"], 0)
        with pytest.raises(RuntimeError, match="before the first request"):
            ctx.serve_add_bank(b.W, b.lo, b.n_time, b.u, b.M, b.q, b.chi, fx.ymin)
        assert ctx.poll(h, b.u.size) is not None
    finally:
        ctx.serve_stop()
    # the context analyses as before once the server has stopped
    r = eb.pe_intrinsic(fx.seg, banks["big"], fx.store, prior=fx.prior_arg, ymin=fx.ymin, n_loud=fx.n_loud,
                        n_random=fx.n_random, seed=0)
    assert np.abs(r["ln_b"] - fx.ln_b).max() <= 1e-5


def test_minimum_idle_time_before_closing_a_worker():
    # one worker slot: bank 'small' needs the slot bank 'big' holds; the big worker was just used, so it is not
    # closed at once (stats after 0.3 s) but once it has been idle for the minimum idle time (1 s)
    fx, ctx, banks, seg = _setup()
    ctx.serve_start(hbm_budget=0, max_workers=1, n_loud=fx.n_loud, n_random=fx.n_random)
    try:
        ctx.serve_set_min_idle(1.0)
        ids = {k: ctx.serve_add_bank(b.W, b.lo, b.n_time, b.u, b.M, b.q, b.chi, fx.ymin) for k, b in banks.items()}
        ctx.poll(ctx.submit(ids["big"], seg["d_H"][0], seg["d_L"][0], seg["sig2_H"], seg["sig2_L"], 0),
                 banks["big"].u.size)
        h = ctx.submit(ids["small"], seg["d_H"][1], seg["d_L"][1], seg["sig2_H"], seg["sig2_L"], 1)
        assert ctx.poll(h, banks["small"].u.size, timeout_us=300000) is None
        assert ctx.serve_stats()["workers_closed"] == 0
        assert ctx.poll(h, banks["small"].u.size) is not None
        st = ctx.serve_stats()
        assert st["workers_closed"] == 1 and st["workers_opened"] == 2
        with pytest.raises(ValueError):
            ctx.serve_set_min_idle(-1.0)
    finally:
        ctx.serve_stop()


def test_concurrent_pollers_read_their_own_error_messages():
    # exm_submit / exm_poll may be called from several host threads (ctypes releases the GIL, so these threads
    # are in the library at the same time): every failed poll's message must be intact and the calling
    # thread's own -- its handle's "has not finished", or the bogus handle it asked for
    import ctypes
    import threading
    fx, ctx, banks, seg = _setup()
    b = banks["small"]
    ctx.serve_start(hbm_budget=0, max_workers=1, n_loud=fx.n_loud, n_random=fx.n_random)
    lib, h = ctx.lib, ctx.h
    bad = []
    try:
        bid = ctx.serve_add_bank(b.W, b.lo, b.n_time, b.u, b.M, b.q, b.chi, fx.ymin)
        handles = [ctx.submit(bid, seg["d_H"][i % 2], seg["d_L"][i % 2], seg["sig2_H"], seg["sig2_L"], i)
                   for i in range(6)]

        def own(hd):
            lnl = np.empty(b.u.size, np.float64)
            lnb = ctypes.c_double()
            while True:
                rc = lib.exm_poll(h, int(hd), 0, lnl.ctypes.data_as(ctypes.c_void_p), ctypes.byref(lnb))
                if rc == _lib.EXM_OK:
                    return
                msg = lib.exm_last_error(h).decode()
                if rc != _lib.EXM_ERR_TIMEOUT or msg != "request %d has not finished" % hd:
                    bad.append((hd, rc, msg))
                    return

        def bogus(k):
            for _ in range(2000):
                rc = lib.exm_poll(h, 10 ** 9 + k, 0, None, None)
                msg = lib.exm_last_error(h).decode()
                if rc != _lib.EXM_ERR_ARG or not msg.startswith("unknown request handle"):
                    bad.append((k, rc, msg))
                    return

        threads = [threading.Thread(target=own, args=(hd,)) for hd in handles]
        threads += [threading.Thread(target=bogus, args=(k,)) for k in range(3)]
        for t in threads:
            t.start()
        for t in threads:
            t.join(timeout=120)
        assert not any(t.is_alive() for t in threads)
        assert not bad, bad[:3]
        st = ctx.serve_stats()
        assert st["served"] == len(handles) and st["failed"] == 0
    finally:
        ctx.serve_stop()
