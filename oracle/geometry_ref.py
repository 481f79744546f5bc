"""ORACLE — test infrastructure only.

Restatement of the reference's host-side geometry input in double precision (JS numbers
are IEEE doubles; the reference stores the result in a Float32Array, grid.js:33):
  naca4_boundary        generateNACA4Boundary        (src/grid.js:38-52)
  rectangular_outer     generateRectangularOuterBoundary (src/grid.js:238-255)
  circular_outer        generateCircularOuterBoundary    (src/grid.js:232-237)
Used to build inputs for the golden fixtures and to check the library's own generators.
"""
from __future__ import annotations

import math

import numpy as np


def naca4_point(t: float, M: int, naca4: int, size: float = 1.0, x_offset: float = 0.0,
                exponent: float = 7 / 5, te_coeff: float = -0.1036):
    """One boundary vertex, t = vertex index (grid.js:38-52).  -0.1036 closes the TE."""
    t /= M / 2
    size *= 2
    thickness = naca4 % 100 / 100
    m = math.floor(naca4 / 1000) / 100
    p = math.floor(naca4 / 100) % 10 / 10

    def thick(s):
        return 5 * thickness * (0.2969 * math.sqrt(s) - 0.126 * s - 0.3516 * s ** 2 + 0.2843 * s ** 3
                                + te_coeff * s ** 4)

    def camber(s):
        return (m / p ** 2) * (2 * p * s - s ** 2) if s < p else (m / (1 - p) ** 2) * ((1 - 2 * p) + 2 * p * s - s ** 2)

    def dcamber(s):
        return ((m / p ** 2) if s < p else (m / (1 - p) ** 2)) * (2 * p - 2 * s)

    def sym(s):
        d = dcamber(s)
        return (thick(s) * -math.sin(math.atan(d)), thick(s) / math.sqrt(1 + d ** 2))

    def upper(s):
        a = sym(s)
        return ((s - 0.5 + a[0]) * size + x_offset, (camber(s) + a[1]) * size)

    def lower(s):
        a = sym(s)
        return ((s - 0.5 - a[0]) * size + x_offset, (camber(s) - a[1]) * size)

    return upper((1 - t) ** exponent) if t <= 1 else lower((t - 1) ** exponent)


def naca4_boundary(M: int, naca4: int, size: float = 1.0, x_offset: float = 0.0, **kw) -> np.ndarray:
    return np.array([naca4_point(i, M, naca4, size, x_offset, **kw) for i in range(M)], dtype=np.float64)


def rectangular_outer(M: int, length_ratio: float = 1.5) -> np.ndarray:
    out = []
    for i in range(M):
        t = i / M
        t = math.fmod(t + 0.125, 1)
        if t < 0.25:
            t *= 4
            out.append((length_ratio, t * 2 - 1))
        elif t < 0.5:
            t = (t - 0.25) * 4
            out.append((((1 - t) * 2 - 1) * length_ratio, 1))
        elif t < 0.75:
            t = (t - 0.5) * 4
            out.append((-length_ratio, (1 - t) * 2 - 1))
        else:
            t = (t - 0.75) * 4
            out.append(((t * 2 - 1) * length_ratio, -1))
    return np.array(out, dtype=np.float64)


def circular_outer(M: int, radius: float = 1.0) -> np.ndarray:
    t = np.arange(M, dtype=np.float64) / M
    return np.stack([radius * np.cos(t * np.pi * 2), radius * np.sin(t * np.pi * 2)], axis=1)


def stretched_guess(body, outer, N: int, first_spacing: float) -> np.ndarray:
    """(N+1, M, 2) float64 initial guess of an O-grid between the body (row 0) and the far
    field (row N): along each column t(j) = h (q^j - 1) / (q - 1) with h = first_spacing / L
    (L the column's length) and q found by bisection so that t(N) = 1; first_spacing <= 0
    gives t = j / N (the reference's linear interpolation, shaders/grid.js:24-27).  This
    restates the library's geometric radial stretching (k_grid_init_d) in double."""
    body = np.asarray(body, np.float64)
    outer = np.asarray(outer, np.float64)
    M = body.shape[0]
    V = np.zeros((N + 1, M, 2))
    V[0], V[N] = body, outer
    j = np.arange(1, N, dtype=np.float64)
    for i in range(M):
        a, b = body[i], outer[i]
        if first_spacing <= 0.0:
            t = j / N
        else:
            L = math.sqrt((b[0] - a[0]) ** 2 + (b[1] - a[1]) ** 2)
            h = first_spacing / L
            lo, hi = 1.0 + 1e-12, 2.0
            if h * N >= 1.0:
                lo, hi = 1e-6, 1.0 - 1e-12
            for _ in range(200):
                q = 0.5 * (lo + hi)
                try:
                    qN = math.pow(q, N)
                except OverflowError:  # q^N beyond double: infinite, as pow returns in C
                    qN = math.inf
                sN = h * (qN - 1.0) / (q - 1.0)
                if (sN > 1.0) == (h * N < 1.0):
                    hi = q
                else:
                    lo = q
            q = 0.5 * (lo + hi)
            qj = np.array([math.pow(q, k) for k in range(1, N)])  # libm pow, as the scalar form
            t = h * (qj - 1.0) / (q - 1.0)
        V[1:N, i, 0] = a[0] * (1.0 - t) + b[0] * t
        V[1:N, i, 1] = a[1] * (1.0 - t) + b[1] * t
    return V
