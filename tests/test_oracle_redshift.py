"""The oracle's restatement of pe_redshift (exmarg/search/pe.py:87-132, 203-257) against the
reference's own outputs (tests/golden/redshift1.npz, produced with the distance function of
exmarg_b200.cosmology standing in for astropy's Planck18)."""

import numpy as np

from exmarg_b200 import cosmology, synth
from oracle import restate
from tests.golden_io import GOLDEN


def load(name="redshift1"):
    import os
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    spec = synth.TableSpec(ntau=int(z["ntau"]), nphif=49, nb=int(z["nb"]), nd=int(z["nd"]))
    fac = (z["fac_M"], z["fac_P"], z["fac_Q"], z["fac_S"])
    s_nodes = z["s_nodes"]
    tables = [synth.gen_table_node(spec, k, s_nodes, int(z["tab_seed"]), fac) for k in range(s_nodes.size)]
    store = synth.MemoryStore(spec, s_nodes, int(z["tab_seed"]), tables=tables)
    seg = dict(d_H=z["d_H"], d_L=z["d_L"], f=z["f"], nu=z["nu"], sig2=z["sig2"], T=float(z["T"]),
               fmin=float(z["fmin"]), fmax=float(z["fmax"]))
    return z, spec, store, seg


def test_source_frame_restatement_matches_reference():
    z, spec, store, seg = load()
    o = restate.pe_redshift(restate.read_segments(seg), z["W"], z["u"], z["bank_rows"][:, 0], int(z["lo"]),
                            int(z["n_time"]), store, cosmology.dl_of_z, zmax=float(z["zmax"]), nz=int(z["nz"]),
                            m1_range=(float(z["m1_lo"]), float(z["m1_hi"])), nm1=int(z["nm1"]),
                            n_loud=int(z["n_loud"]), n_random=int(z["n_random"]), seed=0)
    ref = z["ln_lambda"]
    assert np.array_equal(np.isfinite(o["ln_lambda"]), np.isfinite(ref))
    fin = np.isfinite(ref)
    assert np.abs(o["ln_lambda"][fin] - ref[fin]).max() < 1e-8
    assert np.abs(o["ln_b"] - z["ln_b"]).max() < 1e-9
    assert np.array_equal(o["z"], z["z"]) and np.array_equal(o["m1"], z["m1"])


def test_planck18_restatement_sanity():
    c = cosmology.planck18
    assert abs(c.Om0 + c.Og0 + c.Onu0 + c.Ode0 - 1.0) < 1e-15      # flat
    dl = cosmology.dl_of_z(np.array([1e-4, 1.0]))
    assert abs(dl[0] / (c.hubble_distance * 1e-4) - 1.0) < 1e-3    # Hubble law at small z
    assert 6700.0 < dl[1] < 6900.0                                 # D_L(z = 1) of a Planck-like cosmology
