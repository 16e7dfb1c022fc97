"""The template bank and the matched filter (the contract of exmarg/search/bank.py:17-94).

mass_bank(bank, segments, device) builds W = a e^{i psi0} / D0 on the segments'
frequency bins and u = sum a^2 / sig2_H for every template row (M_det, q, chi), as
the reference does.  device='b200' keeps W on the host and in the context's HBM;
the filter itself runs inside pe_intrinsic (cuFFT + fused kernels), so
trajectories() here is the stage entry point for tests and tools.  device 'cpu'
and 'gpu' return the reference's own MassBank (exmarg.search.mass_bank).

The template profile is exmarg.profiles.profile (lalsuite IMRPhenomXAS) when that
imports, else the closed-form TaylorF2 of exmarg_b200.synth (same signature).
"""

import numpy as np

from . import _lib
from .segments import D0, read_segments


def array_module(device):
    """numpy for 'cpu' and 'b200' host arrays, cupy for 'gpu' (the reference's convention)"""
    if device in ("cpu", "b200"):
        return np
    if device == "gpu":
        import cupy
        return cupy
    raise ValueError("device must be 'cpu', 'gpu' or 'b200'")


def default_profile():
    try:
        from exmarg.profiles import profile   # lalsuite IMRPhenomXAS
        return profile
    except Exception:
        from .synth import profile
        return profile


class MassBank:
    """templates for one frequency grid and noise curve, device 'b200'.

    M, q, chi  (n_template,) detector-frame total mass, mass ratio m2/m1 <= 1, aligned spin
    u          (n_template,) template power sum a^2 / sig2_H at D0
    W          (n_template, n_freq) complex64 a e^{i psi0} (host copy; the device copy
               lives in the analysis context)"""

    def __init__(self, M, q, chi, seg, device="b200", profile=None, W=None, u=None, device_index=0):
        if device != "b200":
            raise ValueError("exmarg_b200.MassBank is the 'b200' bank; use mass_bank() for 'cpu'/'gpu'")
        self.M, self.q, self.chi = np.asarray(M, float), np.asarray(q, float), np.asarray(chi, float)
        self.device, self.xp = device, np
        self.T, self.fmin, self.fmax = seg["T"], seg["fmin"], seg["fmax"]
        self.nu = np.asarray(seg["nu"])
        if not np.all(np.diff(self.nu) == 1):
            raise ValueError("frequency bins must be contiguous")
        self.lo, self.hi = int(self.nu[0]), int(self.nu[-1]) + 1
        self.n_time = 8 * int(self.nu.max())
        if W is None:
            prof = profile or default_profile()
            sig2_H = np.asarray(seg["sig2_H"] if "sig2_H" in seg else seg["sig2"], float)
            W = np.empty((self.M.size, self.nu.size), np.complex64)
            u = np.empty(self.M.size)
            for i in range(self.M.size):
                m1 = self.M[i] / (1.0 + self.q[i])
                m2 = self.M[i] * self.q[i] / (1.0 + self.q[i])
                nu, _, a1, p0 = prof(m1, m2, self.chi[i], self.chi[i], self.T, self.fmin, self.fmax, 1.0)
                j = np.searchsorted(self.nu, nu)
                a = np.zeros(self.nu.size)
                a[j] = a1 / D0
                psi0 = np.zeros(self.nu.size)
                psi0[j] = p0
                W[i] = a * np.exp(1j * psi0)
                u[i] = float((a ** 2 / sig2_H).sum())
        self.W = np.ascontiguousarray(W, np.complex64)
        self.u = np.asarray(u, float)
        self.device_index = device_index

    @property
    def ctx(self):
        c = getattr(self, "_ctx", None)
        return c if c is not None else _lib.context(self.device_index)

    def clone_for(self, ctx):
        """the same bank (host arrays shared) bound to another context, e.g. a child context"""
        seg = dict(T=self.T, fmin=self.fmin, fmax=self.fmax, nu=self.nu)
        b = MassBank(self.M, self.q, self.chi, seg, "b200", W=self.W, u=self.u, device_index=ctx.device)
        b._ctx = ctx
        return b

    def upload(self):
        """make this bank the context's current bank (W copied to HBM)"""
        ctx = self.ctx
        token = _lib.token_of(self)
        if ctx.bank_token != token:
            ctx.bank_set(self.W, self.lo, self.n_time, self.u, self.M, self.q, self.chi)
            ctx.bank_token = token
            ctx.prep_token = None
        return ctx

    def trajectories(self, d, sig2, chunk=1024):
        """matched filter of one segment against every template: dict lqH, phH, lqL, phL
        (n_template, n_time) float32 on the host (exmarg/search/bank.py:56-78).  Needs the
        context prepared for a store (pe_intrinsic, or prepare())."""
        ctx = self.upload()
        if ctx.prep_token is None:
            raise RuntimeError("prepare the context with a store first (pe_intrinsic or exmarg_b200.pe.prepare)")
        return ctx.filter(d["H"][None, :] if np.ndim(d["H"]) == 1 else d["H"], d["L"] if np.ndim(d["L"]) == 1 else d["L"],
                          sig2["H"], sig2["L"])


def mass_bank(bank, segments, device="cpu", profile=None):
    """the template bank: bank is an .npy path or an (n,) / (n, 3) array of rows (M_det[, q, chi])"""
    if device in ("cpu", "gpu"):
        import exmarg.search as ref
        return ref.mass_bank(bank, segments, device)
    if device != "b200":
        raise ValueError("device must be 'cpu', 'gpu' or 'b200'")
    B = np.load(bank) if isinstance(bank, (str, bytes)) or hasattr(bank, "__fspath__") else np.asarray(bank)
    B = np.asarray(B, float)
    if B.ndim == 1:
        B = np.stack([B, np.ones_like(B), np.zeros_like(B)], axis=1)
    seg = read_segments(segments, rows=[0])
    return MassBank(*[np.ascontiguousarray(B[:, i]) for i in range(3)], seg, device, profile=profile)


def from_bank(bank, device_index=0):
    """a 'b200' bank with the W and u of another bank (e.g. the reference's MassBank)"""
    seg = dict(T=bank.T, fmin=bank.fmin, fmax=bank.fmax, nu=bank.nu)
    W = bank.W if isinstance(bank.W, np.ndarray) else bank.W.get()
    return MassBank(bank.M, bank.q, bank.chi, seg, "b200", W=W, u=bank.u, device_index=device_index)
