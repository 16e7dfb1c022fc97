"""Serving: a 256-template request and an 8192-template request give the same ln Lambda alone (the plain
single-segment path, exm_pe_intrinsic) and served together through the native request loop, their segments
on the device at the same time (two workers), bitwise."""

import numpy as np
import pytest

import exmarg_b200 as eb
from exmarg_b200 import synth

pytestmark = pytest.mark.gpu


def test_256_and_8192_templates_alone_and_in_the_mix():
    spec = synth.TableSpec(ntau=43, nb=100, nd=109)
    store = synth.MemoryStore(spec, synth.S_NODES_PROD[10:53:4], 31)          # 11 nodes over the grid
    seg = synth.make_segments(2, 8080, T=8.0, fmax=256.0, snr=(10.0, 30.0), mc=(15.0, 30.0), q=0.8, chi=0.0)
    rows = synth.make_bank(8192, 5)
    big = eb.MassBank(rows[:, 0], rows[:, 1], rows[:, 2], seg, "b200")
    small = eb.MassBank(rows[::32, 0], rows[::32, 1], rows[::32, 2], seg, "b200", W=big.W[::32], u=big.u[::32])
    assert small.u.size == 256
    kw = dict(n_loud=1024, n_random=1024)
    alone = {("small", 0): eb.pe_intrinsic(seg, small, store, rows=[0], **kw),
             ("big", 1): eb.pe_intrinsic(seg, big, store, rows=[1], **kw)}
    ctx = eb.prepare(big, store)
    rd = eb.read_segments(seg)
    ctx.serve_start(max_workers=2, graph=True, **kw)
    try:
        ids = {k: ctx.serve_add_bank(b.W, b.lo, b.n_time, b.u, b.M, b.q, b.chi, 0.1267)
               for k, b in (("small", small), ("big", big))}
        order = [("big", 1), ("small", 0), ("small", 0), ("big", 1), ("small", 0)]
        hs = [(ctx.submit(ids[k], rd["d_H"][e], rd["d_L"][e], rd["sig2_H"], rd["sig2_L"], e), k, e) for k, e in order]
        for h, k, e in hs:
            lnl, lnb = ctx.poll(h, (big if k == "big" else small).u.size)
            ref = alone[(k, e)]
            assert np.array_equal(lnl, ref["ln_lambda"][0]) and lnb == float(ref["ln_b"][0]), (k, e)
        st = ctx.serve_stats()
        assert st["workers_opened"] >= 2 and st["failed"] == 0
    finally:
        ctx.serve_stop()
