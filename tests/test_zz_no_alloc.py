"""exm_gather_noalloc, the gather for callers that cannot allocate device memory during the
call: every input and the output are device buffers the caller owns, and the partial sums
live in a fixed device array of the library.  Its result must equal the allocating entry
point's (exm_gather) on the same trajectories, visited times and slots, call after call."""

import numpy as np
import pytest

import exmarg_b200 as eb
from oracle import restate
from tests.golden_io import Fixture

pytestmark = pytest.mark.gpu

TOL = 1e-9   # the float64 gather contract's tolerance in tests/test_gpu_parity.py


def test_noalloc_gather_matches_gather_two_calls():
    torch = pytest.importorskip("torch")
    fx = Fixture("config1")
    bank = fx.b200_bank()
    ctx = eb.prepare(bank, fx.store, fx.prior_arg, fx.ymin)
    seg = restate.read_segments(fx.seg)
    traj = restate.trajectories(fx.W, {I: seg["d_" + I][0] for I in "HL"}, {I: seg["sig2_" + I] for I in "HL"},
                                fx.lo, fx.n_time, "ref")
    sel, lw = fx.z["sel0"], fx.z["lw0"]
    ctx.set_trajectories(traj)
    ctx.set_times((sel, lw))
    dev = torch.device("cuda", 0)
    d = {k: torch.from_numpy(np.ascontiguousarray(traj[k], np.float32)).to(dev) for k in ("lqH", "phH", "lqL", "phL")}
    d_sel = torch.from_numpy(np.ascontiguousarray(sel, np.int32)).to(dev)
    d_lw = torch.from_numpy(np.ascontiguousarray(lw, np.float32)).to(dev)
    nm, nt = traj["lqH"].shape
    nn = fx.s_nodes.size
    rng = np.random.default_rng(4)
    for call in range(2):
        ids = np.sort(rng.choice(nm, 40 - 13 * call, replace=False)).astype(np.int64)
        ns = 3 - call
        tab = rng.integers(0, nn, size=(ids.size, ns)).astype(np.int64)
        lna = np.log(fx.s_nodes[tab] / fx.u[ids][:, None])
        want = ctx.gather(ids, lna, tab)
        out = torch.full((ns, ids.size), float("nan"), dtype=torch.float64, device=dev)
        d_ids = torch.from_numpy(ids).to(dev)
        d_lna = torch.from_numpy(np.ascontiguousarray(lna)).to(dev)
        d_tab = torch.from_numpy(tab).to(dev)
        torch.cuda.synchronize()
        ctx.gather_noalloc(nm, nt, d["lqH"].data_ptr(), d["phH"].data_ptr(), d["lqL"].data_ptr(), d["phL"].data_ptr(),
                           sel.shape[1], d_sel.data_ptr(), d_lw.data_ptr(), ids.size, ns, d_ids.data_ptr(),
                           d_lna.data_ptr(), d_tab.data_ptr(), out.data_ptr())
        got = out.cpu().numpy()
        assert np.allclose(got, want, rtol=0, atol=TOL), (call, np.abs(got - want).max())


def test_noalloc_gather_rejects_requests_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    fx = Fixture("config1")
    bank = fx.b200_bank()
    ctx = eb.prepare(bank, fx.store, fx.prior_arg, fx.ymin)
    dev = torch.device("cuda", 0)
    buf = torch.zeros(16, dtype=torch.float64, device=dev)
    p = buf.data_ptr()
    nsel = (1 << 20) // fx.spec.ntau + 1      # one lag row more than the scratch holds, one slot
    with pytest.raises(ValueError, match="fixed scratch"):
        ctx.gather_noalloc(4, fx.n_time, p, p, p, p, 0, 0, 0, nsel, 1, p, p, p, p)


def _device_case(torch, fx, ctx):
    seg = restate.read_segments(fx.seg)
    traj = restate.trajectories(fx.W, {I: seg["d_" + I][0] for I in "HL"}, {I: seg["sig2_" + I] for I in "HL"},
                                fx.lo, fx.n_time, "ref")
    dev = torch.device("cuda", 0)
    d = {k: torch.from_numpy(np.ascontiguousarray(traj[k], np.float32)).to(dev) for k in ("lqH", "phH", "lqL", "phL")}
    d["sel"] = torch.from_numpy(np.ascontiguousarray(fx.z["sel0"], np.int32)).to(dev)
    d["lw"] = torch.from_numpy(np.ascontiguousarray(fx.z["lw0"], np.float32)).to(dev)
    return traj, d


def _call(ctx, fx, d, traj, ids, tab, lna, out, sel=None):
    import torch
    torch.cuda.synchronize()          # the inputs were written on torch's stream; the call runs on the context's
    nm, nt = traj["lqH"].shape
    ctx.gather_noalloc(nm, nt, d["lqH"].data_ptr(), d["phH"].data_ptr(), d["lqL"].data_ptr(), d["phL"].data_ptr(),
                       fx.z["sel0"].shape[1], (sel if sel is not None else d["sel"]).data_ptr(), d["lw"].data_ptr(),
                       ids.shape[0], tab.shape[1], ids.data_ptr(), lna.data_ptr(), tab.data_ptr(), out.data_ptr())


def test_noalloc_gather_reports_bad_indices_and_stays_usable():
    # every bad index is caught by the kernel's own checks (the access is skipped) and reported as ValueError
    torch = pytest.importorskip("torch")
    fx = Fixture("config1")
    ctx = eb.prepare(fx.b200_bank(), fx.store, fx.prior_arg, fx.ymin)
    traj, d = _device_case(torch, fx, ctx)
    dev = d["lqH"].device
    nm, nn = traj["lqH"].shape[0], fx.s_nodes.size
    ids = torch.tensor([0, 5, nm - 1], dtype=torch.int64, device=dev)
    tab = torch.zeros((3, 1), dtype=torch.int64, device=dev)
    lna = torch.zeros((3, 1), dtype=torch.float64, device=dev)
    out = torch.zeros((1, 3), dtype=torch.float64, device=dev)
    with pytest.raises(ValueError, match="mass id"):
        _call(ctx, fx, d, traj, torch.tensor([0, nm, 1], dtype=torch.int64, device=dev), tab, lna, out)
    with pytest.raises(ValueError, match="table id"):
        _call(ctx, fx, d, traj, ids, torch.tensor([[0], [nn], [1]], dtype=torch.int64, device=dev), lna, out)
    bad_sel = d["sel"].clone()
    bad_sel[5, 7] = fx.n_time
    with pytest.raises(ValueError, match="visited time"):
        _call(ctx, fx, d, traj, ids, tab, lna, out, sel=bad_sel)
    _call(ctx, fx, d, traj, ids, tab, lna, out)            # and a good call still runs
    assert torch.isfinite(out).all()


def test_noalloc_gather_leaves_device_memory_unchanged():
    torch = pytest.importorskip("torch")
    fx = Fixture("config1")
    ctx = eb.prepare(fx.b200_bank(), fx.store, fx.prior_arg, fx.ymin)
    traj, d = _device_case(torch, fx, ctx)
    dev = d["lqH"].device
    nm, nn = traj["lqH"].shape[0], fx.s_nodes.size
    ids = torch.arange(nm, dtype=torch.int64, device=dev)
    tab = torch.remainder(torch.arange(nm * 2, dtype=torch.int64, device=dev), nn).reshape(nm, 2)
    lna = torch.full((nm, 2), -1.0, dtype=torch.float64, device=dev)
    out = torch.zeros((2, nm), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    _call(ctx, fx, d, traj, ids, tab, lna, out)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info(0)[0]
    _call(ctx, fx, d, traj, ids, tab, lna, out)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free1 == free0
