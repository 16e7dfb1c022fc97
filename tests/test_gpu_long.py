"""16 s segments at 512 Hz (n_time 65536, the longest segment duration the serving mix uses): the device
path against the float64 oracle on a reduced store (21 lags, 100 x 109 tables, six nodes), at the
pe_intrinsic bar."""

import numpy as np
import pytest

import exmarg_b200 as eb
from exmarg_b200 import synth
from oracle import restate

pytestmark = pytest.mark.gpu


def test_16s_segment_matches_fp64_oracle():
    spec = synth.TableSpec(ntau=21, nb=100, nd=109)
    store = synth.MemoryStore(spec, synth.S_NODES_PROD[[20, 26, 32, 38, 44, 50]], 5)
    seg = synth.make_segments(1, 4321, T=16.0, fmax=512.0, snr=20.0, mc=20.0, q=0.8, chi=0.0)
    rows = synth.make_bank(8, 9)
    bank = eb.MassBank(rows[:, 0], rows[:, 1], rows[:, 2], seg, "b200")
    assert bank.n_time == 65536
    res = eb.pe_intrinsic(seg, bank, store, n_loud=1024, n_random=1024)
    o = restate.pe_intrinsic(restate.read_segments(seg), bank.W, bank.u, bank.M, bank.q, bank.chi, bank.lo,
                             bank.n_time, store, n_loud=1024, n_random=1024, seed=0, precision="fp64")
    assert np.all(np.isfinite(res["ln_b"]))
    assert np.abs(res["ln_b"] - o["ln_b"]).max() <= 1e-5
    fin = np.isfinite(o["ln_lambda"])
    assert np.array_equal(fin, np.isfinite(res["ln_lambda"]))
    assert np.abs(res["ln_lambda"][fin] - o["ln_lambda"][fin]).max() <= 1e-4
