"""Golden vectors for the pe_intrinsic path, produced by running the REFERENCE's own CPU
code (exmarg.search: numpy + numba; its table builders scripts/build_tables/w_gpu.py, build_k.py and
build_bd.py, w_gpu.py with numpy standing in for cupy) in a container where its source tree is present.

    python tests/golden/make_golden.py <reference src dir, or - for $EXMARG_REFERENCE_SRC> [case ...]

Each fixture holds the inputs (segments, bank rows, W and u, the store geometry and the
float32 generator factors of its seeded tables) and the reference's outputs (ln_lambda,
ln_b, the visited times of segment 0, and a gather_cpu result).  The tests regenerate
the tables from the stored factors (bit-exact, see exmarg_b200.synth) and compare the
oracle and the B200 path against these outputs; nothing at test time reads the
reference.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from exmarg_b200 import synth  # noqa: E402
from oracle import refimport  # noqa: E402

CASES = {
    # the reduced CPU case: 8 s, analysis band 20-256 Hz (lag unit 1/2048 s, lags +-21),
    # 3 nodes at reduced beta/Delta settings, 64 templates
    "config1": dict(T=8.0, fmax=256.0, ntau=43, nb=100, nd=109, nodes=(14, 24, 34), n_template=64, n_seg=2,
                    snr=15.0, n_loud=1024, n_random=1024, seed_seg=100, seed_bank=3, seed_tab=7, prior="volume"),
    # production lag/table shape (87 lags, 200 x 219), 6 consecutive nodes, 4 s segments
    "prodshape": dict(T=4.0, fmax=512.0, ntau=87, nb=200, nd=219, nodes=tuple(range(20, 26)), n_template=16,
                      n_seg=2, snr=(5.0, 30.0), n_loud=256, n_random=256, seed_seg=500, seed_bank=11, seed_tab=19,
                      prior="volume"),
    # every arrival time walked (n_loud = 0), the tabulated Madau-Dickinson prior, a noise-only segment
    "alltimes_md": dict(T=4.0, fmax=256.0, ntau=43, nb=100, nd=109, nodes=(16, 20, 24, 28), n_template=12,
                        n_seg=2, snr=12.0, noise_only=0.5, n_loud=0, n_random=0, seed_seg=900, seed_bank=5,
                        seed_tab=23, prior="madau-dickinson"),
}


def make(name, c, search):
    spec = synth.TableSpec(ntau=c["ntau"], nphif=49, nb=c["nb"], nd=c["nd"])
    s_nodes = synth.S_NODES_PROD[list(c["nodes"])]
    store = synth.MemoryStore(spec, s_nodes, c["seed_tab"])
    seg = synth.make_segments(c["n_seg"], c["seed_seg"], T=c["T"], fmax=c["fmax"], snr=c["snr"],
                              noise_only=c.get("noise_only", 0.0))
    rows = synth.make_bank(c["n_template"], c["seed_bank"])
    bank = search.mass_bank(rows, seg, "cpu")
    ymin = 0.1267
    if c["prior"] == "madau-dickinson":
        import exmarg.priors as pri
        ymin = float(pri.madau_dickinson_ymin())
    res = search.pe_intrinsic(seg, bank, store, prior=c["prior"], ymin=ymin, n_loud=c["n_loud"],
                              n_random=c["n_random"], seed=0)
    out = dict(d_H=seg["d_H"], d_L=seg["d_L"], f=seg["f"], nu=seg["nu"], sig2=seg["sig2"], T=seg["T"],
               fmin=seg["fmin"], fmax=seg["fmax"], snr=seg["snr"], bank_rows=rows, W=bank.W, u=bank.u,
               lo=bank.lo, n_time=bank.n_time, s_nodes=s_nodes, tab_seed=c["seed_tab"], ntau=spec.ntau,
               nb=spec.nb, nd=spec.nd, ymin=ymin, prior=c["prior"], n_loud=c["n_loud"], n_random=c["n_random"],
               ln_lambda=res["ln_lambda"], ln_b=res["ln_b"])
    M, P, Q, S = spec.factors(s_nodes)
    out.update(fac_M=M, fac_P=P, fac_Q=Q, fac_S=S)
    if c["prior"] == "madau-dickinson":
        import exmarg.priors as pri
        lny, p = pri.distance_density("madau-dickinson")
        out.update(dens_lny=lny, dens_p=p)
    # visited times and one gather_cpu call on segment 0 (its trajectories, all nodes of the first group)
    d = {I: np.asarray(seg["d_" + I][0], complex) for I in "HL"}
    traj = bank.trajectories(d, {I: np.asarray(seg["sig2"], float) for I in "HL"})
    if c["n_loud"] > 0:
        sel, lw = search.gather.select_times(traj, store.tau_idx, c["n_loud"], c["n_random"], 0)
        out.update(sel0=sel, lw0=lw)
        times = (sel, lw)
    else:
        times = None
    ns = min(3, s_nodes.size)
    a = s_nodes[:ns][None, :] / bank.u[:, None]
    lna = np.log(a)
    tab = np.tile(np.arange(ns), (bank.u.size, 1))
    g = search.gather.gather_cpu(traj, dict(T=store.tables[:ns], tau=store.tau_idx, beta=spec.beta,
                                            delta=spec.delta), np.arange(bank.u.size), lna, tab, times)
    out.update(gather_lna=lna, gather_tab=tab, gather_out=g)
    np.savez_compressed(os.path.join(HERE, "%s.npz" % name), **out)
    print(name, "ln_b", res["ln_b"], "size %.1f MB" % (os.path.getsize(os.path.join(HERE, "%s.npz" % name)) / 1e6))


# pe_redshift: an ascending equal-mass, zero-spin bank of detector-frame total masses, 8 s segments, a
# reduced (m1, z) grid.  The reference takes D_L from astropy's Planck18, absent here: a stand-in module
# hands it exmarg_b200.cosmology.dl_of_z (the same restatement the B200 path uses), so these vectors pin
# everything but the distance function itself.
REDSHIFT_CASES = {
    "redshift1": dict(T=8.0, fmax=256.0, ntau=43, nb=100, nd=109, nodes=(10, 14, 18, 22, 26, 30, 34),
                      masses=(12.0, 200.0, 24), n_seg=2, snr=(10.0, 25.0), n_loud=512, n_random=512, seed_seg=1300,
                      seed_tab=29, zmax=4.0, nz=160, m1_range=(3.0, 100.0), nm1=140),
}


def stub_astropy():
    import types
    from exmarg_b200 import cosmology

    class _Quantity:
        def __init__(self, v):
            self.value = v

    class _Planck18:
        @staticmethod
        def luminosity_distance(z):
            return _Quantity(cosmology.dl_of_z(z))

    mod = types.ModuleType("astropy")
    cos = types.ModuleType("astropy.cosmology")
    cos.Planck18 = _Planck18
    mod.cosmology = cos
    sys.modules["astropy"] = mod
    sys.modules["astropy.cosmology"] = cos


def make_redshift(name, c, search):
    stub_astropy()
    spec = synth.TableSpec(ntau=c["ntau"], nphif=49, nb=c["nb"], nd=c["nd"])
    s_nodes = synth.S_NODES_PROD[list(c["nodes"])]
    store = synth.MemoryStore(spec, s_nodes, c["seed_tab"])
    seg = synth.make_segments(c["n_seg"], c["seed_seg"], T=c["T"], fmax=c["fmax"], snr=c["snr"])
    lo_m, hi_m, n_m = c["masses"]
    M = np.geomspace(lo_m, hi_m, n_m)
    rows = np.stack([M, np.ones_like(M), np.zeros_like(M)], axis=1)
    bank = search.mass_bank(rows, seg, "cpu")
    res = search.pe_redshift(seg, bank, store, zmax=c["zmax"], nz=c["nz"], m1_range=c["m1_range"], nm1=c["nm1"],
                             n_loud=c["n_loud"], n_random=c["n_random"], seed=0)
    M_, P, Q, S = spec.factors(s_nodes)
    out = dict(d_H=seg["d_H"], d_L=seg["d_L"], f=seg["f"], nu=seg["nu"], sig2=seg["sig2"], T=seg["T"],
               fmin=seg["fmin"], fmax=seg["fmax"], bank_rows=rows, W=bank.W, u=bank.u, lo=bank.lo,
               n_time=bank.n_time, s_nodes=s_nodes, tab_seed=c["seed_tab"], ntau=spec.ntau, nb=spec.nb, nd=spec.nd,
               ymin=0.1267, n_loud=c["n_loud"], n_random=c["n_random"], zmax=c["zmax"], nz=c["nz"],
               m1_lo=c["m1_range"][0], m1_hi=c["m1_range"][1], nm1=c["nm1"], m1=res["m1"], z=res["z"],
               ln_lambda=res["ln_lambda"], ln_b=res["ln_b"], fac_M=M_, fac_P=P, fac_Q=Q, fac_S=S, prior="volume")
    np.savez_compressed(os.path.join(HERE, "%s.npz" % name), **out)
    print(name, "ln_b", res["ln_b"], "finite", np.isfinite(res["ln_lambda"]).mean(),
          "size %.1f MB" % (os.path.getsize(os.path.join(HERE, "%s.npz" % name)) / 1e6))


# stage 3 of the table build: a synthetic stage-2 store (lnK of a few orders on a small (q1, q2, phi)
# grid) through the reference's scripts/build_tables/build_bd.py build_node, full order and a ladder
BD_CASES = {
    "bd1": dict(nord=9, ntau=3, nq=12, nphi=8, s=1.0, seed=11, ladder=(2, 5, 8)),
}


def synthetic_lnk(c):
    """lnK_n(tau, q1, q2, phi), float32: homogeneous of degree 2n in (q1, q2) (2n ln max(q1, q2) plus a
    function of ln q1 - ln q2), a Poisson-like fall-off in n, smooth in tau and phi, a little noise"""
    rng = np.random.default_rng(c["seed"])
    lnq = np.log(np.geomspace(0.05, 100.0, c["nq"]))
    n = np.arange(c["nord"], dtype=np.float64)[:, None, None, None, None]
    t = np.arange(c["ntau"], dtype=np.float64)[None, :, None, None, None]
    l1 = lnq[None, None, :, None, None]
    l2 = lnq[None, None, None, :, None]
    ph = (2 * np.pi * np.arange(c["nphi"]) / c["nphi"])[None, None, None, None, :]
    from scipy.special import gammaln
    A = (2 * n * np.maximum(l1, l2) + n * (0.4 * np.cos(ph) + 0.1 * t - 0.3 * np.abs(l1 - l2)) - gammaln(n + 1.0)
         + 0.01 * rng.standard_normal((c["nord"], c["ntau"], c["nq"], c["nq"], c["nphi"])))
    return A.astype(np.float32), lnq


def make_bd(name, c, ref_root):
    import importlib.util
    import tempfile
    A, lnq = synthetic_lnk(c)
    tau_idx = np.arange(c["ntau"]) - c["ntau"] // 2
    with tempfile.TemporaryDirectory() as d:
        stem = os.path.join(d, "kstore_n%03d_s%09.3f" % (c["nord"] - 1, c["s"]))
        np.save(stem + ".lnK.npy", A)
        np.savez(stem + ".meta.npz", s_node=c["s"], lnq=lnq, tau_idx=tau_idx)
        os.environ["BD_NMAX_LADDER"] = ",".join(str(v) for v in c["ladder"])
        spec = importlib.util.spec_from_file_location("build_bd", os.path.join(ref_root, "scripts", "build_tables",
                                                                              "build_bd.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        base = os.path.join(d, "bd")
        mod.build_node(stem, base)
        out = dict(lnK=A, lnq=lnq, tau_idx=tau_idx, s=c["s"], ladder=np.array(c["ladder"]))
        for nm in c["ladder"]:
            z = np.load(os.path.join(mod.out_dir(base, nm, c["nord"] - 1), "bd_n%03d_s%09.3f.npz" % (nm, c["s"])))
            out["T%d" % nm] = z["T"]
            out["beta"], out["delta"] = z["beta"], z["delta"]
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, {k: v.shape for k, v in out.items() if hasattr(v, "shape")})


# stage 1 of the table build: the reference's scripts/build_tables/w_gpu.py w_table_s_gpu on a small sky,
# run with numpy in place of cupy and exmarg_b200.wtable's HEALPix pixel centres in place of healpy
W_CASES = {
    "w1": dict(s=(0.5, 3.0, 20.0), n_max=4, nside=2, n_tau=17, chunk=7),
}


def make_w(name, c, ref_root):
    import importlib.util
    import types
    from exmarg_b200 import wtable
    cp = types.ModuleType("cupy")
    cp.__dict__.update({k: getattr(np, k) for k in dir(np) if not k.startswith("_")})
    cp.asnumpy = np.asarray
    cp.cuda = types.SimpleNamespace(Stream=types.SimpleNamespace(null=types.SimpleNamespace(synchronize=lambda: None)))
    sys.modules["cupy"] = cp
    hp = sys.modules.get("healpy") or types.ModuleType("healpy")
    hp.nside2npix = wtable.nside2npix
    hp.pix2ang = wtable.pix2ang
    sys.modules["healpy"] = hp
    spec = importlib.util.spec_from_file_location("w_gpu", os.path.join(ref_root, "scripts", "build_tables", "w_gpu.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    s = np.array(c["s"], float)
    tau, W = mod.w_table_s_gpu(s, s, c["n_max"], n_tau=c["n_tau"], nside=c["nside"], chunk=c["chunk"])
    keys = wtable.keys(c["n_max"])
    out = np.array([[Wj[k] for k in keys] for Wj in W])            # (nodes, keys, tau)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), s=s, n_max=c["n_max"], nside=c["nside"], n_tau=c["n_tau"],
                        tau=tau, W=np.ascontiguousarray(out.transpose(0, 2, 1)))
    print(name, out.shape, float(np.abs(out).max()))


# stage 2 of the table build on the reference's own stage-1 output: node 1 of w1 written as build_w writes it,
# the reference's build_k load_node (delay rebin) and compile_order (every order, on a 12-point magnitude
# grid and 8 phases), then its build_bd on that lnK
K_CASES = {
    "k1": dict(w_case="w1", node=1, nq=12, nphi=8),
}


def make_k(name, c, ref_root):
    import importlib.util
    import tempfile
    from exmarg_b200 import wtable
    z = np.load(os.path.join(HERE, c["w_case"] + ".npz"))
    n_max, s = int(z["n_max"]), float(z["s"][c["node"]])
    with tempfile.TemporaryDirectory() as d:
        stem_w = os.path.join(d, "sladder_n%03d_s%09.3f" % (n_max, s))
        wtable.save_node(stem_w, s, z["tau"], z["W"][c["node"]], n_max, int(z["nside"]))
        spec = importlib.util.spec_from_file_location("build_k", os.path.join(ref_root, "scripts", "build_tables",
                                                                              "build_k.py"))
        bk = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(bk)
        bk.NQ, bk.NPHI = c["nq"], c["nphi"]
        keys, WM, tau_idx = bk.load_node(stem_w)
        lnq = np.log(np.geomspace(bk.QMAX / bk.QSPAN, bk.QMAX, c["nq"]))
        phi_g = np.arange(c["nphi"]) * (2 * np.pi / c["nphi"])
        by_n = {n: [] for n in range(n_max + 1)}
        for j, (n, a, b) in enumerate(keys):
            by_n[int(n)].append((j, int(a), int(b)))
        lnK = np.stack([bk.compile_order(n, s, keys, WM, lnq, by_n, phi_g, tau_idx.size) for n in range(n_max + 1)])
        stem_k = os.path.join(d, "kstore_n%03d_s%09.3f" % (n_max, s))
        np.save(stem_k + ".lnK.npy", lnK)
        np.savez(stem_k + ".meta.npz", s_node=s, lnq=lnq, tau_idx=tau_idx)
        os.environ["BD_NMAX_LADDER"] = ""
        spec = importlib.util.spec_from_file_location("build_bd", os.path.join(ref_root, "scripts", "build_tables",
                                                                              "build_bd.py"))
        bd = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(bd)
        base = os.path.join(d, "bd")
        bd.build_node(stem_k, base)
        out = np.load(os.path.join(base, "bd_n%03d_s%09.3f.npz" % (n_max, s)))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), s=s, n_max=n_max, keys=keys, WM=WM, tau_idx=tau_idx,
                            lnq=lnq, nphi=c["nphi"], lnK=lnK, T=out["T"], beta=out["beta"], delta=out["delta"],
                            W_tau=z["tau"], W=z["W"][c["node"]])
    print(name, lnK.shape, WM.shape)


def main():
    # the reference's src directory: first argument, else $EXMARG_REFERENCE_SRC
    src = refimport.source_dir(sys.argv[1] if len(sys.argv) > 1 and sys.argv[1] != "-" else None)
    if src is None:
        sys.exit("usage: make_golden.py <reference src dir | -> [case ...]  (or set %s)" % refimport.ENV)
    only = sys.argv[2:] if len(sys.argv) > 2 else None
    if only is None or any(n in only for n in list(CASES) + list(REDSHIFT_CASES)):
        search = refimport.import_reference(src)
        for name, c in CASES.items():
            if only is None or name in only:
                make(name, c, search)
        for name, c in REDSHIFT_CASES.items():
            if only is None or name in only:
                make_redshift(name, c, search)
    for name, c in BD_CASES.items():
        if only is None or name in only:
            make_bd(name, c, os.path.dirname(os.path.abspath(src)))
    for name, c in W_CASES.items():
        if only is None or name in only:
            refimport.import_reference(src)          # exmarg on the path, with its stub modules
            make_w(name, c, os.path.dirname(os.path.abspath(src)))
    for name, c in K_CASES.items():
        if only is None or name in only:
            refimport.import_reference(src)
            make_k(name, c, os.path.dirname(os.path.abspath(src)))


if __name__ == "__main__":
    main()
