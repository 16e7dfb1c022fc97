"""The 64-point Gauss-Legendre distance quadrature (an option beside the reference's closed form and
401-point trapezoid, exmarg/search/pe.py:260-286): the library's host rule against numpy's leggauss, and the
oracle's GL weights against the reference's own rules where those are exact or converged."""

import numpy as np
import pytest

from exmarg_b200 import _lib
from oracle import restate
from tests.golden_io import Fixture


@pytest.mark.parametrize("n", [1, 2, 7, 64, 200])
def test_gauss_legendre_rule_matches_numpy(n):
    x, w = _lib.gauss_legendre(n)
    gx, gw = np.polynomial.legendre.leggauss(n)
    assert np.allclose(x, gx, rtol=0, atol=1e-14) and np.allclose(w, gw, rtol=0, atol=1e-14)
    assert abs(w.sum() - 2.0) < 1e-13


def test_gauss_legendre_rejects_bad_n():
    with pytest.raises(ValueError):
        _lib.gauss_legendre(0)


def test_gl64_volume_equals_closed_form():
    # p(y) = 3 ymin^3 y^-4 is smooth on every interval: 64 points reproduce the exact integral (to the
    # rounding of the closed form's differences of exponentials: 4.5e-12 in ln w measured)
    y = np.sort(np.random.default_rng(1).uniform(0.13, 40.0, 30))
    a = restate.distance_weights(y, "volume", 0.1267)
    b = restate.distance_weights(y, "volume", 0.1267, quadrature="gl64")
    assert np.allclose(a, b, rtol=0, atol=1e-10)


def test_gl64_tabulated_close_to_trapezoid():
    lny, p = Fixture("alltimes_md").density         # the reference's Madau-Dickinson table, from a fixture
    y = np.sort(np.exp(np.random.default_rng(2).uniform(lny[0] + 0.1, lny[-1] - 0.1, 25)))
    a = restate.distance_weights(y, "madau-dickinson", 0.1267, (lny, p))
    b = restate.distance_weights(y, "madau-dickinson", 0.1267, (lny, p), quadrature="gl64")
    fin = np.isfinite(a)
    assert np.array_equal(fin, np.isfinite(b))
    assert np.abs(a[fin] - b[fin]).max() < 1e-4     # 2.2e-5 measured: the trapezoid's error
