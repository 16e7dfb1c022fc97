"""Node sharding on the CPU: the host geometry, node ranges and weights agree with the oracle, and
ranks that each supply only their node range's rows (here from the oracle, in place of a GPU) and
exchange them with an all-reduce over gloo get the reference's ln Lambda and ln B on every rank."""

import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from exmarg_b200 import shard
from oracle import restate
from tests.golden_io import Fixture

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def fx_parts():
    fx = Fixture("config1")
    seg = restate.read_segments(fx.seg)
    M, q, chi = (fx.rows[:, i] for i in range(3))
    res = restate.pe_intrinsic(seg, fx.W, fx.u, M, q, chi, fx.lo, fx.n_time, fx.store, prior=fx.prior, ymin=fx.ymin,
                               n_loud=fx.n_loud, n_random=fx.n_random, seed=0, precision="ref", density=fx.density,
                               return_parts=True)
    lam = np.stack([p["lamN"] for p in res["parts"]])
    return fx, lam


def _rows_of(lam, bnode):
    """node_values(seg, k0, k1) of a rank holding nodes k0..k1-1, cut from the whole store's rows"""
    nn = lam.shape[1] - 1

    def node_values(seg, k0, k1):
        out = np.full((lam.shape[0], k1 - k0 + 1, lam.shape[2]), -np.inf)
        out[:, :k1 - k0] = lam[:, k0:k1]
        here = (bnode >= k0) & (bnode < k1)
        out[:, k1 - k0, here] = lam[:, nn, here]
        return out
    return node_values


def _bank(fx):
    from exmarg_b200 import MassBank
    M, q, chi = (fx.rows[:, i] for i in range(3))
    b = MassBank(M, q, chi, fx.seg, "b200", W=fx.W, u=fx.u)
    return b


def test_geometry_and_weights_match_oracle(fx_parts):
    fx, _ = fx_parts
    st = fx.store
    valid, _, y, bnode, _ = restate.node_geometry(st.s, st.alpha_lo, st.alpha_hi, fx.u, fx.ymin)
    v2, y2, b2 = shard.node_geometry(st.s, st.alpha_lo, st.alpha_hi, fx.u, fx.ymin)
    assert np.array_equal(valid, v2) and np.array_equal(y, y2) and np.array_equal(bnode, b2)
    ref = restate.ln_weights(y, fx.prior, fx.ymin, fx.density)
    got = shard.node_weights(st, fx.u, fx.ymin, fx.prior_arg)
    assert np.array_equal(np.isfinite(ref), np.isfinite(got))
    fin = np.isfinite(ref)
    assert np.abs(ref[fin] - got[fin]).max() < 1e-12


def test_node_ranges_cover_the_store(fx_parts):
    fx, _ = fx_parts
    nn = len(fx.store.s)
    for n in range(1, nn + 1):
        r = shard.node_ranges(fx.store, fx.u, fx.ymin, n)
        assert len(r) == n and r[0][0] == 0 and r[-1][1] == nn
        assert all(a < b for a, b in r) and all(r[i][1] == r[i + 1][0] for i in range(n - 1))
    with pytest.raises(ValueError):
        shard.node_ranges(fx.store, fx.u, fx.ymin, nn + 1)


def test_one_rank_matches_reference(fx_parts):
    fx, lam = fx_parts
    _, _, bnode = shard.node_geometry(fx.store.s, fx.store.alpha_lo, fx.store.alpha_hi, fx.u, fx.ymin)
    res = shard.pe_intrinsic_sharded(fx.seg, _bank(fx), fx.store, prior=fx.prior_arg, ymin=fx.ymin,
                                     node_values=_rows_of(lam, bnode))
    assert res["node_ranges"] == [(0, len(fx.store.s))]
    assert np.allclose(res["ln_lambda"], fx.ln_lambda, rtol=0, atol=1e-9)
    assert np.allclose(res["ln_b"], fx.ln_b, rtol=0, atol=1e-9)


def test_one_range_per_rank(fx_parts):
    fx, lam = fx_parts
    _, _, bnode = shard.node_geometry(fx.store.s, fx.store.alpha_lo, fx.store.alpha_hi, fx.u, fx.ymin)
    with pytest.raises(ValueError, match="one node range per rank"):
        shard.pe_intrinsic_sharded(fx.seg, _bank(fx), fx.store, prior=fx.prior_arg, ymin=fx.ymin,
                                   ranges=[(0, 2), (2, len(fx.store.s))], node_values=_rows_of(lam, bnode))


def test_generated_store_is_not_sharded():
    class Generated:
        s = np.array([1.0, 2.0])
        generator = object()
    with pytest.raises(ValueError, match="generated"):
        shard.shard_of(Generated(), 0, 1)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, lam, q):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from exmarg_b200 import shard as sh
        from tests.golden_io import Fixture as F
        fx = F("config1")
        _, _, bnode = sh.node_geometry(fx.store.s, fx.store.alpha_lo, fx.store.alpha_hi, fx.u, fx.ymin)
        res = sh.pe_intrinsic_sharded(fx.seg, _bank(fx), fx.store, prior=fx.prior_arg, ymin=fx.ymin,
                                      node_values=_rows_of(lam, bnode))
        q.put((rank, res["ln_lambda"], res["ln_b"], res["node_ranges"]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_ranks_exchange_rows_over_gloo(fx_parts, world):
    fx, lam = fx_parts
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, lam, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = sorted([q.get(timeout=180) for _ in range(world)], key=lambda g: g[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ranges = got[0][3]
    assert len(ranges) == world and ranges[0][0] == 0 and ranges[-1][1] == len(fx.store.s)
    for rank, ln_lambda, ln_b, r in got:
        assert r == ranges
        assert np.array_equal(ln_lambda, got[0][1]) and np.array_equal(ln_b, got[0][2])
        assert np.allclose(ln_lambda, fx.ln_lambda, rtol=0, atol=1e-9)
        assert np.allclose(ln_b, fx.ln_b, rtol=0, atol=1e-9)


def test_node_ranges_balance_the_work():
    """the ranges' work (pairs plus NODE_WEIGHT a node) differs by at most about one node's work"""
    import numpy as np
    from exmarg_b200 import synth
    s = synth.S_NODES_PROD
    store = type("S", (), {})()
    store.s, store.alpha_lo, store.alpha_hi = s, np.full(s.size, synth.ALPHA[0]), np.full(s.size, synth.ALPHA[-1])
    u = np.geomspace(1.5, 3.0, 300)
    valid, _, bnode = shard.node_geometry(store.s, store.alpha_lo, store.alpha_hi, u, 0.1267)
    work = valid.sum(axis=1) + np.bincount(bnode[bnode >= 0], minlength=s.size)[:s.size] + shard.NODE_WEIGHT
    for n in (2, 3, 4, 8, 16):
        r = shard.node_ranges(store, u, 0.1267, n)
        w = [work[a:b].sum() for a, b in r]
        assert max(w) - min(w) <= 2 * work.max(), (n, w)
