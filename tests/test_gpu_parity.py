"""Parity of the B200 path (libexmarg_b200 through its C ABI) with the reference's outputs
(golden vectors) and with the oracle, stage by stage and end to end."""

import numpy as np
import pytest

import exmarg_b200 as eb
from exmarg_b200 import _lib, synth
from oracle import restate
from tests.golden_io import Fixture

pytestmark = pytest.mark.gpu

CASES = ["config1", "prodshape", "alltimes_md"]
TOL_LNB = 1e-5          # |ln B_b200 - ln B_reference|, float32 tables: 1e-5 absolute
TOL_LNL = 1e-4          # per-template ln Lambda


@pytest.fixture(scope="module", params=CASES)
def fx(request):
    return Fixture(request.param)


def _run(fx, **kw):
    bank = fx.b200_bank()
    return bank, eb.pe_intrinsic(fx.seg, bank, fx.store, prior=fx.prior_arg, ymin=fx.ymin, n_loud=fx.n_loud,
                                 n_random=fx.n_random, seed=0, **kw)


def test_pe_intrinsic_matches_reference(fx):
    _, res = _run(fx)
    assert res["ln_lambda"].shape == fx.ln_lambda.shape
    assert np.all(np.isfinite(res["ln_lambda"]))
    assert np.abs(res["ln_b"] - fx.ln_b).max() <= TOL_LNB
    assert np.abs(res["ln_lambda"] - fx.ln_lambda).max() <= TOL_LNL


def test_pe_intrinsic_against_fp64_oracle(fx):
    _, res = _run(fx)
    seg = restate.read_segments(fx.seg)
    M, q, chi = (fx.rows[:, i] for i in range(3))
    o = restate.pe_intrinsic(seg, fx.W, fx.u, M, q, chi, fx.lo, fx.n_time, fx.store, prior=fx.prior, ymin=fx.ymin,
                             n_loud=fx.n_loud, n_random=fx.n_random, seed=0, precision="fp64", density=fx.density)
    assert np.abs(res["ln_b"] - o["ln_b"]).max() <= TOL_LNB


def test_pe_intrinsic_deterministic(fx):
    _, a = _run(fx)
    _, b = _run(fx)
    assert np.array_equal(a["ln_lambda"], b["ln_lambda"]) and np.array_equal(a["ln_b"], b["ln_b"])


def test_rows_subset_matches_full_run(fx):
    _, full = _run(fx)
    _, one = _run(fx, rows=[1])
    assert np.array_equal(one["ln_lambda"][0], full["ln_lambda"][1])


def _ref_traj(fx):
    seg = restate.read_segments(fx.seg)
    return restate.trajectories(fx.W, {I: seg["d_" + I][0] for I in "HL"}, {I: seg["sig2_" + I] for I in "HL"},
                                fx.lo, fx.n_time, "ref")


def test_filter_matches_oracle(fx):
    bank = fx.b200_bank()
    ctx = eb.prepare(bank, fx.store, fx.prior_arg, fx.ymin)
    seg = restate.read_segments(fx.seg)
    tr = ctx.filter(seg["d_H"][:1], seg["d_L"][:1], seg["sig2_H"], seg["sig2_L"])
    ref = _ref_traj(fx)
    for I in "HL":
        big = ref["lq" + I] > ref["lq" + I].max(axis=1, keepdims=True) - 3.0   # the loud part of each series
        assert np.abs(tr["lq" + I] - ref["lq" + I])[big].max() < 2e-5
        d = np.abs(tr["ph" + I] - ref["ph" + I])
        d = np.minimum(d, 2 * np.pi - d)
        assert d[big].max() < 2e-5


def test_select_times_on_same_trajectories(fx):
    if fx.n_loud == 0:
        pytest.skip("every arrival time is walked")
    bank = fx.b200_bank()
    ctx = eb.prepare(bank, fx.store, fx.prior_arg, fx.ymin)
    ref = _ref_traj(fx)
    ctx.set_trajectories(ref)
    sel, lw = ctx.select_times(0, fx.n_loud, fx.n_random)
    # index work: every template visits exactly the reference's times with the reference's weights
    assert np.array_equal(sel, fx.z["sel0"])
    assert np.array_equal(lw, fx.z["lw0"])


def test_score_exp_is_numpys():
    from tests.test_npexp import _same_bits, sample_inputs
    x = sample_inputs()
    with np.errstate(over="ignore", invalid="ignore"):
        ref = np.exp(x)
    ctx = _lib.Context(0)
    try:
        got = ctx.np_exp32(x)
    finally:
        ctx.close()
    bad = ~_same_bits(got, ref)
    assert not bad.any(), list(zip(x[bad][:5], got[bad][:5], ref[bad][:5]))


def test_select_times_tie_takes_earliest():
    # scores tied at the n_loud-th place: numpy's argpartition leaves the choice among them unspecified;
    # the device takes the earliest tied times (the strictly larger scores are always all taken)
    fx = Fixture("config1")
    bank = fx.b200_bank()
    ctx = eb.prepare(bank, fx.store, fx.prior_arg, fx.ymin)
    nm, nt, K, S = fx.u.size, fx.n_time, 64, 32
    rng = np.random.default_rng(5)
    lqL = rng.uniform(-3.0, 3.0, (nm, nt)).astype(np.float32)
    order = np.argsort(-lqL, axis=1, kind="stable")
    tied = order[:, K - 3:K + 4]                                  # 7 times share the K-th largest value
    np.put_along_axis(lqL, tied, np.take_along_axis(lqL, order[:, K - 3:K - 2], axis=1), axis=1)
    traj = dict(lqH=np.full((nm, nt), -40.0, np.float32), phH=np.zeros((nm, nt), np.float32), lqL=lqL,
                phL=np.zeros((nm, nt), np.float32))
    ctx.set_trajectories(traj)
    sel, lw = ctx.select_times(3, K, S)
    for m in range(nm):
        loud = np.sort(sel[m][lw[m] == 0])
        want = np.sort(np.concatenate([order[m, :K - 3], np.sort(tied[m])[:3]]))
        assert np.array_equal(loud, want)


def test_gather_contract_float64(fx):
    bank = fx.b200_bank()
    ctx = eb.prepare(bank, fx.store, fx.prior_arg, fx.ymin)
    ctx.set_trajectories(_ref_traj(fx))
    ctx.set_times((fx.z["sel0"], fx.z["lw0"]) if "sel0" in fx.z else None)
    out = ctx.gather(np.arange(fx.u.size), fx.z["gather_lna"], fx.z["gather_tab"])
    assert np.allclose(out, fx.z["gather_out"], rtol=0, atol=1e-9)


def test_node_values_plane_gather(fx):
    bank = fx.b200_bank()
    ctx = eb.prepare(bank, fx.store, fx.prior_arg, fx.ymin)
    traj = _ref_traj(fx)
    times = (fx.z["sel0"], fx.z["lw0"]) if "sel0" in fx.z else None
    ctx.set_trajectories(traj)
    ctx.set_times(times)
    lam = ctx.node_values(fx.s_nodes.size)
    geom = restate.node_geometry(fx.store.s, fx.store.alpha_lo, fx.store.alpha_hi, fx.u, fx.ymin)
    groups = [list(range(g, min(g + 6, fx.s_nodes.size))) for g in range(0, fx.s_nodes.size, 6)]
    ref = restate.node_values(traj, fx.store, geom, groups, times)
    fin = np.isfinite(ref)
    assert np.array_equal(fin, np.isfinite(lam))
    assert np.abs(lam[fin] - ref[fin]).max() < 2e-5


def test_device_generator_bit_exact():
    spec = synth.TableSpec(ntau=43, nphif=49, nb=100, nd=109)
    s = synth.S_NODES_PROD[10:13]
    ctx = _lib.Context(0)
    try:
        ctx.store_init(3, spec.shape, spec.tau_idx, spec.beta[0], spec.beta[1] - spec.beta[0], spec.delta[0],
                       spec.delta[1] - spec.delta[0])
        M, P, Q, S = spec.factors(s)
        for k in range(3):
            ctx.store_generate_node(k, s[k], 0.16, 4e4, M, P, Q, S[k], 99)
        for k in range(3):
            assert np.array_equal(ctx.store_get_node(k, spec.shape), synth.gen_table_node(spec, k, s, 99))
    finally:
        ctx.close()


def test_errors_are_reported():
    fx = Fixture("config1")
    bank = fx.b200_bank()
    with pytest.raises(ValueError):
        eb.pe_intrinsic(fx.seg, bank, fx.store, n_loud=16, n_random=0)      # division by zero in the reference
    with pytest.raises(ValueError):
        eb.pe_intrinsic(fx.seg, bank, fx.store, n_loud=fx.n_time)            # high <= 0
    with pytest.raises(ValueError):
        eb.pe_intrinsic(fx.seg, bank, fx.store, prior="flat")
    bad = dict(fx.seg, d_H=fx.seg["d_H"][:, :-1], d_L=fx.seg["d_L"][:, :-1])
    with pytest.raises(ValueError):
        eb.pe_intrinsic(bad, bank, fx.store)
    # a store whose only node lies below every template's amplitude range (a = s/u < ymin^2)
    one = synth.MemoryStore(fx.spec, np.array([1e-6]), 1, tables=fx.store.tables[:1])
    with pytest.raises(ValueError, match="fewer than two store nodes"):
        eb.pe_intrinsic(fx.seg, bank, one)
    # the context is still usable after the errors
    res = eb.pe_intrinsic(fx.seg, bank, fx.store, n_loud=fx.n_loud, n_random=fx.n_random)
    assert np.abs(res["ln_b"] - fx.ln_b).max() <= TOL_LNB


@pytest.mark.parametrize("name", ["config1", "alltimes_md"])
def test_gl64_quadrature_matches_oracle(name):
    # the 64-point Gauss-Legendre distance quadrature on the device against the oracle's (numpy's rule)
    fx = Fixture(name)
    bank = fx.b200_bank()
    res = eb.pe_intrinsic(fx.seg, bank, fx.store, prior=fx.prior_arg, ymin=fx.ymin, n_loud=fx.n_loud,
                          n_random=fx.n_random, seed=0, quadrature="gl64")
    seg = restate.read_segments(fx.seg)
    M, q, chi = (fx.rows[:, i] for i in range(3))
    o = restate.pe_intrinsic(seg, fx.W, fx.u, M, q, chi, fx.lo, fx.n_time, fx.store, prior=fx.prior, ymin=fx.ymin,
                             n_loud=fx.n_loud, n_random=fx.n_random, seed=0, precision="ref", density=fx.density,
                             quadrature="gl64")
    assert np.abs(res["ln_b"] - o["ln_b"]).max() <= TOL_LNB
    assert np.abs(res["ln_lambda"] - o["ln_lambda"]).max() <= TOL_LNL
