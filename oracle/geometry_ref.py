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
