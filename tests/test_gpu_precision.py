"""16-bit tables (float16 with a per-node power-of-two scale, bfloat16): the device quantizer is
bit-exact with its host restatement, the analysis on 16-bit tables matches the oracle run on the
same quantized values (the float32 path's bar), and the error the quantization itself brings
into ln B, against the reference on the float32 tables, stays inside the stated bounds."""

import numpy as np
import pytest

import exmarg_b200 as eb
from exmarg_b200 import _lib, synth
from oracle import restate
from tests.golden_io import Fixture

pytestmark = pytest.mark.gpu

CASES = ["config1", "prodshape", "alltimes_md"]
DTYPES = ["f16", "bf16"]
TOL_IMPL = 1e-5                          # |ln B| device vs oracle on the same 16-bit values
TOL_QUANT = {"f16": 5e-3, "bf16": 2e-2}  # |ln B| on 16-bit tables vs the reference on float32 tables


@pytest.mark.parametrize("dt", DTYPES)
def test_device_quantizer_bit_exact(dt):
    spec = synth.TableSpec(ntau=7, nphif=49, nb=90, nd=171)
    s = synth.S_NODES_PROD[20:23]
    M, P, Q, S = spec.factors(s)
    ctx = _lib.Context(0)
    try:
        ctx.store_init(3, spec.shape, spec.tau_idx, spec.beta[0], spec.beta[1] - spec.beta[0], spec.delta[0],
                       spec.delta[1] - spec.delta[0], eb.store.TABLE_DTYPES[dt])
        host = [synth.gen_table_node(spec, k, s, 5) for k in range(3)]
        ctx.store_set_node(0, s[0], 0.16, 4e4, host[0])                      # uploaded float32, quantized
        for k in (1, 2):
            ctx.store_generate_node(k, s[k], 0.16, 4e4, M, P, Q, S[k], 5)    # generated, quantized
        for k in range(3):
            assert np.array_equal(ctx.store_get_node(k, spec.shape), eb.quantize_table(host[k], dt)[0])
    finally:
        ctx.close()


def _oracle_quantized(fx, dt):
    seg = restate.read_segments(fx.seg)
    M, q, chi = (fx.rows[:, i] for i in range(3))
    st = synth.MemoryStore(fx.spec, fx.s_nodes, 0, tables=[eb.quantize_table(T, dt)[0] for T in fx.store.tables])
    return restate.pe_intrinsic(seg, fx.W, fx.u, M, q, chi, fx.lo, fx.n_time, st, prior=fx.prior, ymin=fx.ymin,
                                n_loud=fx.n_loud, n_random=fx.n_random, seed=0, precision="fp64",
                                density=fx.density), st


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("name", CASES)
def test_pe_intrinsic_16bit(name, dt):
    fx = Fixture(name)
    bank = fx.b200_bank()
    store16 = eb.with_table_dtype(fx.store, dt)
    res = eb.pe_intrinsic(fx.seg, bank, store16, prior=fx.prior_arg, ymin=fx.ymin, n_loud=fx.n_loud,
                          n_random=fx.n_random, seed=0)
    o, _ = _oracle_quantized(fx, dt)
    assert np.abs(res["ln_b"] - o["ln_b"]).max() <= TOL_IMPL
    assert np.abs(res["ln_lambda"] - o["ln_lambda"]).max() <= 1e-4
    assert np.abs(res["ln_b"] - fx.ln_b).max() <= TOL_QUANT[dt]


@pytest.mark.parametrize("dt", DTYPES)
def test_gather_contract_16bit(dt):
    fx = Fixture("config1")
    bank = fx.b200_bank()
    store16 = eb.with_table_dtype(fx.store, dt)
    ctx = eb.prepare(bank, store16, fx.prior_arg, fx.ymin)
    seg = restate.read_segments(fx.seg)
    traj = restate.trajectories(fx.W, {I: seg["d_" + I][0] for I in "HL"}, {I: seg["sig2_" + I] for I in "HL"},
                                fx.lo, fx.n_time, "ref")
    times = (fx.z["sel0"], fx.z["lw0"])
    ctx.set_trajectories(traj)
    ctx.set_times(times)
    out = ctx.gather(np.arange(fx.u.size), fx.z["gather_lna"], fx.z["gather_tab"])
    qt = [eb.quantize_table(T, dt)[0] for T in fx.store.tables]
    ref = restate.gather(traj, qt, np.arange(fx.u.size), fx.z["gather_lna"], fx.z["gather_tab"], fx.spec.beta,
                         fx.spec.delta, fx.spec.tau_idx, times)
    assert np.allclose(out, ref, rtol=0, atol=1e-9)
