"""Velocity-space quadratures for the DUGKS step (the `constant/Xis` and
`constant/weights` inputs of a dugksFoam case).

Two 1-D rules are provided, as the reference generator offers them
(src/scripts/setDV.py:83-138):

* ``gauss_hermite_half_range(C, n)`` -- the half-range Gauss-Hermite rule of
  setDV.py:83-112.  The nodes of the rule for the weight exp(-x^2) on
  [0, inf) are the eigenvalues of the symmetric tridiagonal Jacobi matrix
  built from the recurrence coefficients (alpha_i, beta_i) of the monic
  orthogonal polynomials for that weight (Golub-Welsch).  The coefficients
  follow the nonlinear recurrence written at setDV.py:90-98.  The half-range
  rule is mirrored to (-inf, inf), the weights are multiplied by exp(x^2) so
  that they integrate f(x) rather than f(x) exp(-x^2), and both are scaled by
  the most probable speed C (setDV.py:106-111).
* ``newton_cotes(xi_max, n)`` -- the compound Newton-Cotes (Boole) rule of
  setDV.py:114-138 on [-xi_max, xi_max], n = 4Z + 1 points.

``tensor_product(xis, weights, D)`` builds the D-dimensional set in the
order fvDVM::initialiseDV uses (src/fvDVM/fvDVM/fvDVM.C:293-374): x fastest,
then y, then z; xi components beyond D are zero and the weight of a DV is
the product of its 1-D weights.
"""
from __future__ import annotations

import math

import numpy as np


def _half_range_recurrence(m: int) -> tuple[np.ndarray, np.ndarray]:
    """Recurrence coefficients (alpha, beta) of the monic polynomials
    orthogonal for exp(-x^2) on [0, inf), as setDV.py:90-98 computes them."""
    alpha = np.zeros(m)
    beta = np.zeros(m)
    sqrt_pi = math.sqrt(math.pi)
    alpha[0] = 1.0 / sqrt_pi
    if m > 1:
        alpha[1] = 2.0 / sqrt_pi / (math.pi - 2.0)
        beta[1] = alpha[0] / (alpha[0] + alpha[1]) / 2.0
    for i in range(2, m):
        beta[i] = (i - 1) + 0.5 - beta[i - 1] - alpha[i - 1] ** 2
        alpha[i] = (i * i / 4.0 / beta[i] - beta[i - 1] - 0.5) / alpha[i - 1] - alpha[i - 1]
    return alpha, beta


def gauss_hermite_half_range(C: float, n: int) -> tuple[np.ndarray, np.ndarray]:
    """Full-range 1-D DV set built from the half-range Gauss-Hermite rule.

    ``n`` is the total number of nodes (even, >= 6, setDV.py:146-150);
    ``C`` the scaling speed (sqrt(2 R T) for the usual choice).
    Returns (xis, weights), ascending xis.
    """
    if n % 2 != 0 or n < 6:
        raise ValueError("number of discrete velocities must be even and at least 6")
    m = n // 2
    alpha, beta = _half_range_recurrence(m)
    off = np.sqrt(beta[1:m])
    jac = np.diag(alpha) + np.diag(off, 1) + np.diag(off, -1)
    # a general (non-symmetric) eigen-solver, as setDV.py:103 uses; the
    # weights of the outermost nodes are ill-conditioned in the eigenvector
    # and a symmetric solver moves them by ~1e-10 relative
    nodes, vecs = np.linalg.eig(jac)
    nodes = np.real(nodes)
    vecs = np.real(vecs)
    w = vecs[0, :] * vecs[0, :] * math.sqrt(math.pi) / 2.0
    order = np.argsort(nodes)
    nodes = nodes[order]
    w = w[order]
    xis = np.concatenate((-nodes[::-1], nodes))
    weights = np.concatenate((w[::-1], w))
    weights = weights * np.exp(xis ** 2) * C
    xis = xis * C
    return xis, weights


def newton_cotes(xi_max: float, n: int) -> tuple[np.ndarray, np.ndarray]:
    """Compound Newton-Cotes (Boole's rule) on [-xi_max, xi_max] with
    n = 4Z + 1 equally spaced points (setDV.py:114-138)."""
    if n % 4 != 1 or n < 5:
        raise ValueError("number of points must be 4*Z + 1")
    xi_min = -xi_max
    dv = (xi_max - xi_min) / (n - 1)
    xis = xi_min + dv * np.arange(n, dtype=np.float64)
    w = np.zeros(n)
    for i in range((n - 1) // 4):
        w[4 * i + 0] = 14.0 / 90 * 4
        w[4 * i + 1] = 32.0 / 90 * 4
        w[4 * i + 2] = 12.0 / 90 * 4
        w[4 * i + 3] = 32.0 / 90 * 4
    w[0] = 7.0 / 90 * 4
    w[n - 1] = 7.0 / 90 * 4
    return xis, dv * w


def tensor_product(xis: np.ndarray, weights: np.ndarray, D: int) -> tuple[np.ndarray, np.ndarray]:
    """D-dimensional DV set: returns (xi [Nv,3], w [Nv]) with index
    i = (iz*n + iy)*n + ix, as fvDVM.C:304-321 (3-D) and :335-349 (2-D)."""
    n = len(xis)
    if D == 3:
        iz, iy, ix = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
        ix, iy, iz = ix.ravel(), iy.ravel(), iz.ravel()
        xi = np.stack([xis[ix], xis[iy], xis[iz]], axis=1)
        w = weights[iz] * weights[iy] * weights[ix]
    elif D == 2:
        iy, ix = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
        ix, iy = ix.ravel(), iy.ravel()
        xi = np.stack([xis[ix], xis[iy], np.zeros(n * n)], axis=1)
        w = weights[iy] * weights[ix] * 1
    elif D == 1:
        xi = np.stack([xis, np.zeros(n), np.zeros(n)], axis=1)
        w = weights * 1 * 1
    else:
        raise ValueError("D must be 1, 2 or 3")
    return np.ascontiguousarray(xi, dtype=np.float64), np.ascontiguousarray(w, dtype=np.float64)


def write_foam_list(path: str, obj: str, values: np.ndarray) -> None:
    """Write a 1-D scalar list in the layout setDV.py:67-81 writes."""
    with open(path, "w") as f:
        f.write("FoamFile\n{\n    version     2.0;\n    format      ascii;\n"
                "    class       dictionary;\n    location    \"constant\";\n"
                f"    object      {obj};\n}}\n")
        f.write(f"{len(values)}\n(\n")
        for v in values:
            f.write("% 18.15e\n" % v)
        f.write(");\n")
