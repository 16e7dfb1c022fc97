"""The offline table build, stage 1 (the contract of scripts/build_tables/w_gpu.py and build_w.py): the
GORFs W^(n)_ab(tau) at fixed distance at every node of s, on the B200.

    W_j(tau, (n, a, b)) = scale_j(n) sum_pix dep(pix, tau) sum_{psi, chi} w_q e^{-s_j (|R1|^2 + |R2|^2)}
                          cos((a - b)(arg R1 - arg R2)) (|R1|/sqrt2)^(a+b) (|R2|/sqrt2)^(2n-a-b)

over the HEALPix sky (RING pixel centres), the polarization angle psi (2 n_max + 3 points) and cos(inclination)
chi (Gauss-Legendre, n_max + 3 points); R_I = A_+(chi) F+_I + i chi Fx_I the detector responses, dep the linear
deposit of each pixel's H-L delay on the tau grid, scale_j(n) = s_j^n 2^n / n!.

The host side here builds the geometry (pixel centres, antenna patterns, delays and their deposit weights,
the quadrature, the key list and the scales); exm_w_build (csrc/wtable.cu) runs the quadrature on the device
in float64: per pixel the responses and power ladders, then for each phase class m = a - b one fused
register-tiled FP64 GEMM over the quadrature points whose second operand (the monomials) is generated in
shared memory, deposited on the two delay bins of the pixel.
"""

import os
import time

import numpy as np

from . import _lib

# the detectors (LAL vertex positions and arm directions, as exmarg/detectors.py:10-15 gives them)
C_LIGHT = 299792458.0
X = {"H": np.array([-2.16141492636e6, -3.83469517889e6, 4.60035022664e6]),
     "L": np.array([-7.42760447238e4, -5.49628371971e6, 3.22425701744e6])}
U = {"H": np.array([-0.22389266154, 0.79983062746, 0.55690487831]),
     "L": np.array([-0.95457412153, -0.14158077340, -0.26218911324])}
V = {"H": np.array([-0.91397818574, 0.02609403989, -0.40492342125]),
     "L": np.array([0.29774156894, -0.48791033647, -0.82054461286])}
D = {I: 0.5 * (np.outer(U[I], U[I]) - np.outer(V[I], V[I])) for I in "HL"}

N_MAX, NSIDE, N_TAU = 120, 32, 257          # the settings of the published tables (build_w.py:26)


def nside2npix(nside):
    return 12 * int(nside) ** 2


def pix2ang(nside, ipix):
    """(theta, phi) of the centres of HEALPix RING-scheme pixels (Gorski et al. 2005, ApJ 622, 759, sect. 4)"""
    nside = int(nside)
    p = np.asarray(ipix, np.int64)
    npix = nside2npix(nside)
    ncap = 2 * nside * (nside - 1)
    z = np.empty(p.shape)
    phi = np.empty(p.shape)
    north = p < ncap
    south = p >= npix - ncap
    belt = ~north & ~south
    if north.any():
        q = p[north]
        i = (1 + np.floor(np.sqrt(1.0 + 2.0 * q)).astype(np.int64)) // 2
        i = np.where(2 * i * (i - 1) > q, i - 1, i)                     # guard the square root's rounding
        i = np.where(2 * (i + 1) * i <= q, i + 1, i)
        j = q + 1 - 2 * i * (i - 1)
        z[north] = 1.0 - i * i * 4.0 / npix
        phi[north] = (j - 0.5) * np.pi / (2.0 * i)
    if belt.any():
        q = p[belt] - ncap
        i = q // (4 * nside) + nside
        j = q % (4 * nside) + 1
        f = 0.5 * (1 + ((i + nside) & 1))
        z[belt] = (2 * nside - i) * (8.0 * nside / npix)
        phi[belt] = (j - f) * np.pi / (2.0 * nside)
    if south.any():
        q = npix - p[south]
        i = (1 + np.floor(np.sqrt(2.0 * q - 1.0)).astype(np.int64)) // 2
        i = np.where(2 * i * (i - 1) >= q, i - 1, i)
        i = np.where(2 * (i + 1) * i < q, i + 1, i)
        j = 4 * i + 1 - (q - 2 * i * (i - 1))
        z[south] = -1.0 + i * i * 4.0 / npix
        phi[south] = (j - 0.5) * np.pi / (2.0 * i)
    return np.arccos(np.clip(z, -1.0, 1.0)), phi


def basis(theta, phi):
    """n_hat, theta_hat, phi_hat (last axis the vector component), exmarg/detectors.py:21-32"""
    st, ct, sp, cp = np.sin(theta), np.cos(theta), np.sin(phi), np.cos(phi)
    n = np.stack([st * cp, st * sp, ct], axis=-1)
    th = np.stack([ct * cp, ct * sp, -st], axis=-1)
    ph = np.stack([-sp, cp, np.zeros_like(st)], axis=-1)
    return n, th, ph


def antenna(I, theta, phi):
    """F+ and Fx of detector I at polarization angle 0 (exmarg/detectors.py:35-49)"""
    _, th, ph = basis(theta, phi)
    ep = th[..., :, None] * th[..., None, :] - ph[..., :, None] * ph[..., None, :]
    ex = th[..., :, None] * ph[..., None, :] + ph[..., :, None] * th[..., None, :]
    return np.einsum("ab,...ab->...", D[I], ep), np.einsum("ab,...ab->...", D[I], ex)


def quadrature(n_max, n_psi=None, n_chi=None):
    """psi grid, chi Gauss-Legendre nodes, combined weights (exmarg/tables.py:42-50)"""
    n_psi = 2 * n_max + 3 if n_psi is None else n_psi
    n_chi = n_max + 3 if n_chi is None else n_chi
    psi = np.arange(n_psi) * (np.pi / n_psi)
    cg, cw = np.polynomial.legendre.leggauss(n_chi)
    return psi, cg, cw / 2.0 / n_psi


def tau_grid(n_tau):
    """the delay grid over the H-L light time (exmarg/tables.py:136-146)"""
    tau_max = np.linalg.norm(X["H"] - X["L"]) / C_LIGHT
    return np.linspace(-tau_max, tau_max, n_tau)


def deposit(tau, theta, phi, npix):
    """per pixel: the lower delay bin j0 and the weights (1 - f, f) / npix of bins j0, j0 + 1
    (exmarg/tables.py:123-133 on an ascending tau grid)"""
    t_del = (basis(theta, phi)[0] @ (X["H"] - X["L"])) / C_LIGHT
    dtau = tau[1] - tau[0]
    g = (t_del - tau[0]) / dtau
    j0 = np.clip(np.floor(g).astype(np.int64), 0, tau.size - 2)
    fr = g - j0
    return j0.astype(np.int32), np.stack([(1.0 - fr) / npix, fr / npix], axis=1)


def keys(n_max):
    """(n, a, b), b <= a, in the reference's order (exmarg/tables.py:36-39)"""
    return [(n, a, b) for n in range(n_max + 1) for a in range(n + 1) for b in range(a + 1)]


def scales(s_nodes, n_max):
    """(n_nodes, n_keys) s^n / n! 2^n, its logarithm capped at 700 (w_gpu.py:146-151)"""
    from scipy.special import gammaln
    n_key = np.array([k[0] for k in keys(n_max)], float)
    s = np.atleast_1d(np.asarray(s_nodes, float))
    ln_scale = n_key[None, :] * np.log(s)[:, None] - gammaln(n_key + 1.0)[None, :] + n_key[None, :] * np.log(2.0)
    return np.exp(np.minimum(ln_scale, 700.0))


def geometry(nside, n_max, n_tau, pixels=None):
    """the inputs of exm_w_build: per pixel float32 (F+_H, Fx_H, F+_L, Fx_L) at psi = 0, the delay bin and
    deposit weights; the quadrature in the types the responses use (float32 cos 2psi, sin 2psi, A+ and chi,
    float64 weights); the tau grid"""
    npix = nside2npix(nside)
    pix = np.arange(npix) if pixels is None else np.asarray(pixels)
    th, ph = pix2ang(nside, pix)
    resp = np.empty((pix.size, 4), np.float32)
    for j, I in enumerate("HL"):
        fp, fx = antenna(I, th, ph)
        resp[:, 2 * j] = fp.astype(np.float32)
        resp[:, 2 * j + 1] = fx.astype(np.float32)
    psi, cg, wq = quadrature(n_max)
    tau = tau_grid(n_tau)
    j0, w = deposit(tau, th, ph, npix)
    return dict(resp=resp, j0=j0, w=w, c2p=np.cos(2 * psi).astype(np.float32), s2p=np.sin(2 * psi).astype(np.float32),
                ap=(0.5 * (1 + cg ** 2)).astype(np.float32), cg=cg.astype(np.float32), wq=np.asarray(wq, np.float64),
                tau=tau, npix=npix)


def w_table(s_nodes, n_max=N_MAX, nside=NSIDE, n_tau=N_TAU, pixels=None, device=0, ctx=None):
    """tau (n_tau,), W (n_nodes, n_tau, n_keys) float32 over keys(n_max), stats.  pixels: a subset of the
    sky (for timing); the deposit weights still divide by the whole sky's pixel count."""
    g = geometry(nside, n_max, n_tau, pixels)
    sc = scales(s_nodes, n_max)
    ctx = ctx or _lib.context(device)
    W, ms = ctx.w_build(np.atleast_1d(np.asarray(s_nodes, np.float64)), n_max, g, sc)
    if not np.isfinite(W).all():
        raise FloatingPointError("conditional W table non-finite")
    return g["tau"], W, {"kernel_ms": ms[0], "ms": ms[1]}


def save_node(stem, s_node, tau, Wj, n_max, nside):
    """one node as build_w.py:30-37 writes it: the (a >= b) keys as float32 .W.npy and a .meta.npz"""
    ks = keys(n_max)
    np.save(str(stem) + ".W.npy", np.ascontiguousarray(Wj.T, np.float32))
    np.savez(str(stem) + ".meta.npz", tau=tau.astype(np.float32), keys=np.array(ks, np.int16), norm="taylor_off1",
             s_node=float(s_node), n_max=n_max, nside=nside, shape=np.array([len(ks), tau.size]))


def build_w(out, s_nodes, n_max=N_MAX, nside=NSIDE, n_tau=N_TAU, device=0):
    """every node of s_nodes: <out>/sladder_n<n_max>_s<s>.W.npy and .meta.npz, and manifest.npz (build_w.py)"""
    os.makedirs(out, exist_ok=True)
    t0 = time.time()
    tau, W, _ = w_table(s_nodes, n_max, nside, n_tau, device=device)
    seconds = time.time() - t0
    for s, Wj in zip(np.atleast_1d(s_nodes), W):
        save_node(os.path.join(out, "sladder_n%03d_s%09.3f" % (n_max, s)), s, tau, Wj, n_max, nside)
    np.savez(os.path.join(out, "manifest.npz"), s_nodes=np.asarray(s_nodes), n_max=n_max, nside=nside, n_tau=n_tau,
             s_min=float(np.min(s_nodes)), s_max=float(np.max(s_nodes)), built_s=seconds)
    return seconds


def main(argv=None):
    """python -m exmarg_b200.wtable <out_dir> [node indices]   the W tables of the nodes (build_w.py)
    Nodes: the 53 of the published store (exmarg_b200.synth.S_NODES_PROD), or --s-grid <npz with s_nodes>."""
    import argparse
    ap = argparse.ArgumentParser(prog="python -m exmarg_b200.wtable", description=main.__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("out_dir")
    ap.add_argument("nodes", nargs="*", type=int)
    ap.add_argument("--s-grid", default=None)
    ap.add_argument("--n-max", type=int, default=N_MAX)
    ap.add_argument("--nside", type=int, default=NSIDE)
    ap.add_argument("--n-tau", type=int, default=N_TAU)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    if args.s_grid:
        s_all = np.load(args.s_grid)["s_nodes"]
    else:
        from .synth import S_NODES_PROD as s_all
    s_nodes = np.asarray(s_all)[args.nodes or list(range(len(s_all)))]
    if s_nodes.size > 64:
        raise SystemExit("at most 64 nodes per build")
    seconds = build_w(args.out_dir, s_nodes, args.n_max, args.nside, args.n_tau, args.device)
    print("%d nodes in %.0f s, written to %s" % (s_nodes.size, seconds, args.out_dir), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
