"""The segments an analysis reads (the contract of exmarg/search/segments.py:11-54).

read_segments takes an npz path, a loaded npz or a dict with d_H, d_L (n_segment,
n_freq) complex frequency-domain data, f, nu (contiguous integer bins f T), sig2 or
sig2_H / sig2_L (noise variance per bin), T, fmin and fmax, and returns d_H, d_L as
complex128 and sig2_H, sig2_L as float64 with the selected rows.
"""

import os

import numpy as np

D0 = 10410.0    # Mpc: reference distance of the stores, y = D0 / D_L


def read_segments(segments, rows=None):
    path = isinstance(segments, (str, bytes, os.PathLike))
    z = np.load(segments, mmap_mode="r") if path else segments
    dH = z["d_H"]
    n = np.asarray(dH).shape[0] if not path else dH.shape[0]
    rows = np.arange(n) if rows is None else np.asarray(rows, int)
    out = {"rows": rows, "f": np.asarray(z["f"], float), "nu": np.asarray(z["nu"], np.int64),
           "T": float(z["T"]), "fmin": float(z["fmin"]), "fmax": float(z["fmax"])}
    keys = z.files if hasattr(z, "files") else list(z.keys())
    for I in "HL":
        out["d_" + I] = np.asarray(np.asarray(z["d_" + I])[rows]).astype(complex)
        key = "sig2_" + I if "sig2_" + I in keys else "sig2"
        out["sig2_" + I] = np.asarray(z[key], float)
    return out
