"""Velocity quadrature: the restatement against the reference generator's
own outputs (tests/golden/quadrature_setdv.json, made by running
setDV.py's dvGH/dvNC) and the reference demo's constant/Xis, weights."""
import math

import numpy as np

import golden_cases
from dugks_b200 import quadrature


def test_gauss_hermite_matches_setdv_bitwise():
    g = golden_cases.setdv_quadrature()
    C = g["C"]
    for n, ref in g["GH"].items():
        x, w = quadrature.gauss_hermite_half_range(C, int(n))
        assert np.array_equal(x, np.array(ref["xis"])), n
        assert np.array_equal(w, np.array(ref["weights"])), n


def test_newton_cotes_matches_setdv_bitwise():
    g = golden_cases.setdv_quadrature()
    for key, ref in g["NC"].items():
        xm, n = key.split("_")
        x, w = quadrature.newton_cotes(float(xm), int(n))
        assert np.array_equal(x, np.array(ref["xis"])), key
        assert np.array_equal(w, np.array(ref["weights"])), key


def test_demo_quadrature_files():
    # the demo's files were written with 16 significant digits by an older
    # numpy/LAPACK; nodes agree to ~2e-12 and weights to ~1e-10 (the
    # exp(x^2) factor amplifies the node difference)
    z = golden_cases.demo_cavity(flatten=False)
    x, w = quadrature.gauss_hermite_half_range(golden_cases.setdv_quadrature()["C"], 28)
    assert np.max(np.abs(x - z.xis) / np.abs(z.xis)) < 1e-11
    assert np.max(np.abs(w - z.weights) / z.weights) < 1e-9


def test_gauss_hermite_known_answers():
    C = 337.0
    for n in (8, 16, 28):
        x, w = quadrature.gauss_hermite_half_range(C, n)
        # integral of exp(-x^2/C^2) and of its second moment
        assert abs(np.sum(w * np.exp(-(x / C) ** 2)) / (math.sqrt(math.pi) * C) - 1) < 1e-13
        assert abs(np.sum(w * x ** 2 * np.exp(-(x / C) ** 2)) / (math.sqrt(math.pi) * C ** 3 / 2) - 1) < 1e-12
        assert np.allclose(x, -x[::-1]) and np.allclose(w, w[::-1])


def test_tensor_product_order():
    x = np.array([-2.0, -1.0, 1.0, 2.0])
    w = np.array([0.1, 0.2, 0.3, 0.4])
    xi, ww = quadrature.tensor_product(x, w, 3)
    i = (2 * 4 + 1) * 4 + 3  # iz=2, iy=1, ix=3
    assert np.array_equal(xi[i], [2.0, -1.0, 1.0])
    assert ww[i] == w[2] * w[1] * w[3]
    xi2, ww2 = quadrature.tensor_product(x, w, 2)
    assert np.array_equal(xi2[1 * 4 + 2], [1.0, -1.0, 0.0]) and ww2[1 * 4 + 2] == w[1] * w[2]
