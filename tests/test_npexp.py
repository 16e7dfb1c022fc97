"""The selection score's exp (exmarg/search/gather.py:407: numpy's float32 np.exp) restated in C
(oracle/npexp.c, the host twin of the device's exm_np_expf) and checked bit for bit against np.exp.

The restatement was also compared with np.exp on all 2^32 float32 inputs (no difference); this test
covers every float32 of magnitude in [1, 16) -- where 2 ln|z| decides rankings -- every 97th bit
pattern of the whole line, and the edges (overflow, underflow into subnormals and zero, inf, NaN)."""

import ctypes

import numpy as np

from oracle import build_oracle


def _restated(x):
    lib = ctypes.CDLL(build_oracle.build())
    lib.oracle_npexp32_array.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]
    lib.oracle_npexp32_array.restype = None
    x = np.ascontiguousarray(x, np.float32)
    y = np.empty_like(x)
    lib.oracle_npexp32_array(x.ctypes.data, y.ctypes.data, x.size)
    return y


def _same_bits(a, b):
    return (a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))


def sample_inputs():
    lo, hi = np.float32(1.0).view(np.uint32), np.float32(16.0).view(np.uint32)
    dense = np.arange(lo, hi, dtype=np.uint32).view(np.float32)
    dense = np.concatenate([dense, -dense])
    sparse = np.arange(0, 1 << 32, 97, dtype=np.uint64).astype(np.uint32).view(np.float32)
    edges = np.array([88.72283935546875, 88.7228317, 88.72284, -103.97208404541015625, -103.972076, -87.3, -87.4,
                      -88.0, -100.0, -103.9, 0.0, -0.0, np.inf, -np.inf, np.nan, 1e-30, -1e-30], np.float32)
    return np.concatenate([dense, sparse, edges])


def test_restated_exp_is_numpys_bit_for_bit():
    x = sample_inputs()
    with np.errstate(over="ignore", invalid="ignore"):
        ref = np.exp(x)
    got = _restated(x)
    bad = ~_same_bits(got, ref)
    assert not bad.any(), list(zip(x[bad][:5], got[bad][:5], ref[bad][:5]))


def test_correct_rounding_would_not_do():
    # the reason the restatement exists: a correctly rounded exp differs from numpy's in the last bit
    x = np.arange(np.float32(1.0).view(np.uint32), np.float32(1.0).view(np.uint32) + 200000,
                  dtype=np.uint32).view(np.float32)
    exact = np.exp(x.astype(np.float64)).astype(np.float32)
    assert (exact != np.exp(x)).any()
