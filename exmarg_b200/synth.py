"""Seeded synthetic inputs of the production shape: templates, segments, tables.

Nothing here is on the measured path; it builds the inputs that the tests and the
benchmark feed to it.

* `profile`    a closed-form 3.5PN TaylorF2 inspiral with aligned spins, with the
               return signature of the reference's template profile
               (exmarg/profiles.py:26-47: bin indices, frequencies, amplitude,
               phase).  lalsuite's IMRPhenomXAS is absent here; both the
               reference path and this package consume the same W, so parity
               does not depend on which waveform fills it.
* `psd`        an analytic aLIGO-design-like one-sided PSD (the zero-detuned
               high-power fit of Ajith 2011, arXiv:1107.1267 Eq. 4.7).
* `make_segments`  frequency-domain H1/L1 segments in the dict layout that
               `read_segments` takes (exmarg/search/segments.py:11-54), with
               Gaussian noise of variance sig2 = T S / 2 per bin and one
               injected TaylorF2 signal at a chosen network SNR (the model of
               exmarg/pp.py:38-72; sky, orientation, phase and arrival time
               drawn from the seed).
* `make_bank`  a seeded Latin hypercube over (chirp mass, q, chi_eff), returned
               as rows (M_det, q, chi) like the reference's banks.
* tables       per-node lnS tables T[tau, phi+, beta, Delta] in the reference's
               bd_*.npz layout (scripts/build_tables/build_bd.py:83-84).  The
               values are lnS = ln I0(2 sqrt(x)) * P(phi) * Q(tau) - s/4 with
               x = e^beta (1 + e^(2 Delta)) / 2, plus a hashed perturbation of
               at most 2^-7.  That shape has the real dynamic range (about 4e4
               in the loud corner, about -1e3 at the top node for noise).  The
               per-(beta, Delta) factor is evaluated once in float64 and
               rounded to float32; every later step is one IEEE float32
               operation in a fixed order, so `gen_table_node` (numpy) and the
               device generator in the CUDA library give bit-identical tables.
"""

import os

import numpy as np
from scipy.special import i0e

D0 = 10410.0                    # Mpc: reference distance of the stores, y = D0 / D_L
T_SUN = 4.925490947641267e-06   # G Msun / c^3 (s)
C_LIGHT = 299792458.0
MPC_M = 3.085677581491367e22
EULER_GAMMA = 0.5772156649015329
NPHI = 96


# ----------------------------------------------------------------------------- noise

def psd(f, f_low=10.0):
    """one-sided PSD (1/Hz) of the aLIGO zero-detuned high-power fit; inf below f_low"""
    f = np.asarray(f, float)
    x = np.where(f > 0, f, 1.0) / 215.0
    s = 1e-49 * (x ** -4.14 - 5.0 * x ** -2 + 111.0 * (1.0 - x ** 2 + 0.5 * x ** 4) / (1.0 + 0.5 * x ** 2))
    return np.where(f >= f_low, s, np.inf)


def freq_bins(T, fmin, fmax):
    """integer bins nu = f T with fmin <= f <= fmax"""
    return np.arange(int(np.ceil(fmin * T)), int(np.floor(fmax * T)) + 1)


# ----------------------------------------------------------------------------- waveform

def _taylorf2_phase(f, m1, m2, chi):
    """3.5PN TaylorF2 phase Psi(f) (stationary phase), aligned equal spins chi on both bodies.

    Coefficients: non-spinning terms to 3.5PN (Buonanno et al. 2009, arXiv:0907.0700,
    Eq. 3.18), leading spin-orbit (1.5PN) and spin-spin (2PN) terms.  Constant and
    linear-in-f pieces are dropped: the phase and arrival-time marginalisations absorb
    them."""
    M = m1 + m2
    eta = m1 * m2 / M ** 2
    v = (np.pi * M * T_SUN * f) ** (1.0 / 3.0)
    beta = chi * (113.0 - 76.0 * eta) / 12.0
    sigma = eta * chi * chi * 474.0 / 48.0
    p2 = 3715.0 / 756.0 + 55.0 * eta / 9.0
    p3 = -16.0 * np.pi + 4.0 * beta
    p4 = 15293365.0 / 508032.0 + 27145.0 * eta / 504.0 + 3085.0 * eta ** 2 / 72.0 - 10.0 * sigma
    p5l = 3.0 * np.pi * (38645.0 / 756.0 - 65.0 * eta / 9.0)          # coefficient of ln v at v^5
    p6 = (11583231236531.0 / 4694215680.0 - 640.0 * np.pi ** 2 / 3.0 - 6848.0 * EULER_GAMMA / 21.0
          + (-15737765635.0 / 3048192.0 + 2255.0 * np.pi ** 2 / 12.0) * eta
          + 76055.0 * eta ** 2 / 1728.0 - 127825.0 * eta ** 3 / 1296.0)
    p6l = -6848.0 / 21.0
    p7 = np.pi * (77096675.0 / 254016.0 + 378515.0 * eta / 1512.0 - 74045.0 * eta ** 2 / 756.0)
    lv = np.log(v)
    series = (1.0 + p2 * v ** 2 + p3 * v ** 3 + p4 * v ** 4 + p5l * lv * v ** 5
              + (p6 + p6l * (np.log(4.0) + lv)) * v ** 6 + p7 * v ** 7)
    return 3.0 / (128.0 * eta * v ** 5) * series


def profile(m1, m2, s1z, s2z, T, fmin, fmax, D0_mpc):
    """TaylorF2 template on the segment's bins: (nu, f, a, psi0), face-on h+ at distance D0_mpc.

    Same return convention as the reference's profile (exmarg/profiles.py:26-47): only
    bins with a > 0 are returned (the inspiral stops at the Schwarzschild ISCO)."""
    chi = 0.5 * (s1z + s2z)
    nu = freq_bins(T, fmin, fmax)
    f = nu / T
    M = m1 + m2
    mc = M * (m1 * m2 / M ** 2) ** 0.6
    f_isco = 1.0 / (6.0 ** 1.5 * np.pi * M * T_SUN)
    amp = np.sqrt(5.0 / 24.0) * np.pi ** (-2.0 / 3.0) * (mc * T_SUN) ** (5.0 / 6.0) * C_LIGHT / (D0_mpc * MPC_M)
    a = np.where(f <= f_isco, amp * f ** (-7.0 / 6.0), 0.0)
    psi0 = -_taylorf2_phase(f, m1, m2, chi)
    keep = a > 0
    return nu[keep], f[keep], a[keep], psi0[keep]


# ----------------------------------------------------------------------------- detectors

_EARTH_R = 6.371e6
# site latitude, longitude and x-arm / y-arm azimuths (deg, from north through east)
_SITES = {"H": (46.455, -119.408, 324.0, 54.0), "L": (30.563, -90.774, 252.3, 162.3)}


def _site(I):
    lat, lon, ax, ay = np.radians(_SITES[I])
    up = np.array([np.cos(lat) * np.cos(lon), np.cos(lat) * np.sin(lon), np.sin(lat)])
    east = np.array([-np.sin(lon), np.cos(lon), 0.0])
    north = np.cross(up, east)
    arm = lambda az: np.sin(az) * east + np.cos(az) * north
    u, v = arm(ax), arm(ay)
    return _EARTH_R * up, 0.5 * (np.outer(u, u) - np.outer(v, v))


def antenna(I, theta, phi, psi):
    """F+, Fx of site I for a source at polar angle theta, azimuth phi, polarisation psi"""
    _, d = _site(I)
    n = np.array([np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), np.cos(theta)])
    ex = np.array([np.cos(theta) * np.cos(phi), np.cos(theta) * np.sin(phi), -np.sin(theta)])
    ey = np.array([-np.sin(phi), np.cos(phi), 0.0])
    c2, s2 = np.cos(2 * psi), np.sin(2 * psi)
    p = np.outer(ex, ex) - np.outer(ey, ey)
    x = np.outer(ex, ey) + np.outer(ey, ex)
    return float(np.sum(d * (p * c2 - x * s2))), float(np.sum(d * (p * s2 + x * c2))), n


# ----------------------------------------------------------------------------- segments

def chirp_to_total(mc, q):
    """detector-frame total mass of chirp mass mc and mass ratio q = m2/m1 <= 1"""
    return mc * (1.0 + q) ** 1.2 / q ** 0.6


def make_segments(n, seed, T=8.0, fmin=20.0, fmax=512.0, snr=15.0, noise_only=0.0,
                  mc=25.0, q=0.8, chi=0.1, dtype=np.complex128):
    """n seeded segments, each in its own Gaussian noise, with one injection.

    snr        network optimal SNR: a number, or (lo, hi) to draw it uniformly per segment
    noise_only fraction of segments without a signal (drawn from the seed)
    mc, q, chi injection parameters: numbers, or (lo, hi) ranges drawn per segment
    returns the segment dict of read_segments plus 'snr' and 'truth' (mc, q, chi, y)."""
    nu = freq_bins(T, fmin, fmax)
    f = nu / T
    sig2 = T * psd(f) / 2.0
    dH = np.empty((n, nu.size), dtype)
    dL = np.empty((n, nu.size), dtype)
    snrs = np.zeros(n)
    truth = np.zeros((n, 4))
    pick = lambda rng, v: rng.uniform(*v) if isinstance(v, (tuple, list)) else float(v)
    xH, _ = _site("H")
    xL, _ = _site("L")
    for k in range(n):
        rng = np.random.default_rng(seed + k)
        mck, qk, chik, rho = pick(rng, mc), pick(rng, q), pick(rng, chi), pick(rng, snr)
        if rng.uniform() < noise_only:
            rho = 0.0
        theta, phi = np.arccos(rng.uniform(-1, 1)), rng.uniform(0, 2 * np.pi)
        psi, cosi = rng.uniform(0, np.pi), rng.uniform(-1, 1)
        phase, t0 = rng.uniform(0, 2 * np.pi), rng.uniform(0.1 * T, 0.9 * T)
        M = chirp_to_total(mck, qk)
        m1, m2 = M / (1 + qk), M * qk / (1 + qk)
        nu_t, _, a1, p0 = profile(m1, m2, chik, chik, T, fmin, fmax, 1.0)
        h = np.zeros(nu.size, complex)
        h[np.searchsorted(nu, nu_t)] = a1 / D0 * np.exp(1j * p0)
        sig = {}
        rho2 = 0.0
        for I, xI in (("H", xH), ("L", xL)):
            Fp, Fx, nhat = antenna(I, theta, phi, psi)
            R = complex(0.5 * (1 + cosi ** 2) * Fp + 1j * cosi * Fx)
            tau = nhat @ (xI - xL) / C_LIGHT
            sig[I] = R * np.exp(-1j * phase) * h * np.exp(-2j * np.pi * f * (t0 + tau))
            rho2 += 2.0 * np.sum(np.abs(sig[I]) ** 2 / sig2)
        y = rho / np.sqrt(rho2) if rho2 > 0 else 0.0
        for I, d in (("H", dH), ("L", dL)):
            g = rng.standard_normal((2, nu.size))
            d[k] = np.sqrt(sig2 / 2.0) * (g[0] + 1j * g[1]) + y * sig[I]
        snrs[k] = rho
        truth[k] = mck, qk, chik, y
    return dict(d_H=dH, d_L=dL, f=f, nu=nu, sig2=sig2, T=float(T), fmin=float(fmin), fmax=float(fmax),
                snr=snrs, truth=truth)


def make_bank(n, seed, mc=(10.0, 40.0), q=(0.25, 1.0), chi=(-0.5, 0.5)):
    """(n, 3) rows (M_det, q, chi): a seeded Latin hypercube over (chirp mass, q, chi)"""
    rng = np.random.default_rng(seed)
    cols = []
    for lo, hi in (mc, q, chi):
        u = (rng.permutation(n) + rng.uniform(size=n)) / n
        cols.append(lo + (hi - lo) * u)
    mcv, qv, cv = cols
    return np.stack([chirp_to_total(mcv, qv), qv, cv], axis=1)


# ----------------------------------------------------------------------------- tables

# the 53 signal-power nodes of the published store: logarithmic from s_min to 4000 (data/tables/s_grid.npz:
# s_min, s_max, n_nodes; equal to its s_nodes within 2.3e-15)
S_NODES_PROD = np.geomspace(0.004264528739608287, 4000.0, 53)
ALPHA = np.geomspace(0.16, 4.0e4, 30)                                    # amplitude axis of each node


class TableSpec:
    """geometry of a store: lags, phase planes and the (beta, Delta) grids (shared by every node).

    The production shape is ntau = 87 (lags -43..43 in FFT order), nphif = 49,
    nb = 200 and nd = 219 on the grids of scripts/build_tables/build_bd.py:56-62."""

    def __init__(self, ntau=87, nphif=49, nb=200, nd=219, nq=110):
        self.ntau, self.nphif, self.nb, self.nd = ntau, nphif, nb, nd
        lnq = np.log(np.geomspace(0.05, 100.0, nq))
        dlq = float(lnq[1] - lnq[0])
        half = ntau // 2
        self.tau_idx = np.concatenate([np.arange(0, half + 1), np.arange(-half, 0)]).astype(np.int64)
        self.beta = np.log(ALPHA[0]) + 2.0 * lnq[0] + 2.0 * dlq * np.arange(nb)
        c = nd // 2
        self.delta = dlq * (np.arange(nd) - c)
        self.lnq = lnq

    @property
    def shape(self):
        return (self.ntau, self.nphif, self.nb, self.nd)

    def factors(self, s_nodes):
        """float32 factors: M (nb, nd), P (nphif,), Q (ntau,), S (n_node,)"""
        x = np.exp(self.beta)[:, None] * (1.0 + np.exp(2.0 * self.delta))[None, :] / 2.0
        z = 2.0 * np.sqrt(x)
        M = (np.log(i0e(z)) + z).astype(np.float32)
        P = (0.6 + 0.4 * np.cos(np.arange(self.nphif) * np.pi / (self.nphif - 1))).astype(np.float32)
        Q = (0.8 + 0.2 * np.cos(np.pi * self.tau_idx / (self.ntau // 2 + 1))).astype(np.float32)
        S = (np.asarray(s_nodes, float) / 4.0).astype(np.float32)
        return M, P, Q, S


def _mix32(h):
    """32-bit integer finaliser (multiply-xorshift), on uint32 numpy arrays"""
    h = h ^ (h >> np.uint32(16))
    h = h * np.uint32(0x7FEB352D)
    h = h ^ (h >> np.uint32(15))
    h = h * np.uint32(0x846CA68B)
    return h ^ (h >> np.uint32(16))


def table_hash(seed, k, r, c, b, d):
    """uint32 hash of a table cell (broadcasting); the device generator computes the same"""
    u = np.uint32
    with np.errstate(over="ignore"):
        h = (u(seed) * u(0x9E3779B1)) ^ (np.asarray(k, np.uint32) * u(0x85EBCA77))
        h = _mix32(h ^ (np.asarray(r, np.uint32) * u(0xC2B2AE3D)))
        h = _mix32(h ^ (np.asarray(c, np.uint32) * u(0x27D4EB2F)))
        h = _mix32(h ^ (np.asarray(b, np.uint32) * u(0x165667B1)))
        h = _mix32(h ^ (np.asarray(d, np.uint32) * u(0xD3A2646C)))
    return h


def gen_table_node(spec, k, s_nodes, seed, factors=None, rows=None):
    """float32 table (ntau, nphif, nb, nd) of node k (or the lag rows `rows` of it)"""
    M, P, Q, S = factors if factors is not None else spec.factors(s_nodes)
    rr = np.arange(spec.ntau) if rows is None else np.asarray(rows)
    out = np.empty((rr.size, spec.nphif, spec.nb, spec.nd), np.float32)
    c = np.arange(spec.nphif, dtype=np.uint32)[:, None, None]
    b = np.arange(spec.nb, dtype=np.uint32)[None, :, None]
    d = np.arange(spec.nd, dtype=np.uint32)[None, None, :]
    scale = np.float32(2.0 ** -22)
    for i, r in enumerate(rr):
        v = M[None, :, :] * P[:, None, None]
        v = v * Q[r]
        v = v - S[k]
        h = table_hash(seed, k, r, c, b, d)
        pert = ((h & np.uint32(0xFFFF)).astype(np.int32) - 32768).astype(np.float32) * scale
        out[i] = v + pert
    return out


def write_store(path, spec, s_nodes, seed, n_max=120):
    """write one bd_*.npz per node, uncompressed, in the reference's layout"""
    os.makedirs(path, exist_ok=True)
    fac = spec.factors(s_nodes)
    files = []
    for k, s in enumerate(s_nodes):
        T = gen_table_node(spec, k, s_nodes, seed, fac)
        fn = os.path.join(path, "bd_n%03d_s%09.3f.npz" % (n_max, s))
        np.savez(fn, T=T, beta=spec.beta, delta=spec.delta, tau_idx=spec.tau_idx, lnq=spec.lnq,
                 alpha=ALPHA, s_node=float(s), u_node=float(s), n_max=n_max, nphif=spec.nphif,
                 norm="synthetic")
        files.append(fn)
    return files


class MemoryStore:
    """a store held in memory with the fields of the reference's RedshiftStore
    (exmarg/search/store.py:77-87)"""

    def __init__(self, spec, s_nodes, seed, tables=None, n_max=120, table_dtype="f32"):
        self.spec = spec
        self.table_dtype = table_dtype
        self.s = np.asarray(s_nodes, float)
        self.alpha_lo = np.full(self.s.size, ALPHA[0])
        self.alpha_hi = np.full(self.s.size, ALPHA[-1])
        self.beta = [spec.beta] * self.s.size
        self.delta = [spec.delta] * self.s.size
        self.tau_idx = spec.tau_idx
        self.n_max = n_max
        self.seed = seed
        if tables is None:
            fac = spec.factors(self.s)
            tables = [gen_table_node(spec, k, self.s, seed, fac) for k in range(self.s.size)]
        self.tables = tables
