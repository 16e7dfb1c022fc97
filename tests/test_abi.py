"""The C ABI: the library loads, exports every symbol the header declares, and its host-only
parts (the numpy-compatible RNG) work without a GPU."""

import os
import re

import numpy as np
import pytest

from exmarg_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "exmarg_b200.h")


def declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"EXM_API[^;(]*?\b(exm_\w+)\s*\(", src)))


def test_header_declares_what_the_binding_uses():
    assert sorted(_lib.SYMBOLS) == declared()


def test_every_declared_symbol_is_exported():
    lib = _lib.load()
    missing = [s for s in declared() if not hasattr(lib, s)]
    assert missing == []
    assert lib.exm_version() >= 10000


@pytest.mark.parametrize("seed,high,n", [(0, 31744, 20000), (5, 7, 3000), (2 ** 33 + 1, 1000003, 5000),
                                         (12345, 3, 50), (77, 2 ** 31 + 11, 4000), (9, 1, 10)])
def test_rng_matches_numpy(seed, high, n):
    assert np.array_equal(_lib.rng_integers(seed, high, n), np.random.default_rng(seed).integers(0, high, n))


def test_rng_rejects_bad_arguments():
    with pytest.raises(ValueError):
        _lib.rng_integers(1, 0, 5)


def test_no_cpu_fallback_without_gpu():
    import subprocess
    import sys
    code = ("import exmarg_b200\n"
            "try:\n    exmarg_b200.context(0)\nexcept RuntimeError as e:\n    print('RAISED')\n"
            "else:\n    print('OPENED')\n")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         cwd=os.path.dirname(os.path.dirname(HEADER)))
    import torch
    if torch.cuda.is_available():
        assert "OPENED" in out.stdout
    else:
        assert "RAISED" in out.stdout        # no device: the call fails, nothing falls back to the CPU
