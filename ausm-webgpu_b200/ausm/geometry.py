"""Host geometry front end: airfoil .dat files and analytic bodies.

The .dat reader follows the reference's parser (src/airfoilDatParser.js):
  extract_blocks    numeric lines grouped by blank lines, point-count headers dropped (:29-57)
  parse_dat         Lednicer (2+ blocks starting near x=0) or Selig (split at min x) (:67-105)
  build_spline      centripetal Catmull-Rom through the contour with phantom end points,
                    arc-length parameter, Barry-Goldman evaluation (:116-236)
  sample_airfoil    n points at logit-clustered parameters (a = 5), scaled to a chord of
                    2*scale centred at x_offset (:280-293)
Analytic bodies and outer boundaries come from the library (ausm_naca4_points,
ausm_outer_points) so that every host shares one implementation.
"""
from __future__ import annotations

import ctypes as C
import math
import re

import numpy as np

from . import _lib

_NUM = re.compile(r"^[+-]?(?:\d+\.?\d*(?:[eE][+-]?\d+)?|\.\d+(?:[eE][+-]?\d+)?|Infinity)")


def _parse_float(tok: str) -> float:
    """JavaScript parseFloat: the longest numeric prefix, NaN when there is none."""
    m = _NUM.match(tok)
    if not m:
        return math.nan
    s = m.group(0)
    return float(s.replace("Infinity", "inf"))


def extract_blocks(text: str):
    blocks, cur = [], []
    for line in text.split("\n"):
        t = line.strip()
        if not t:
            if cur:
                blocks.append(cur)
                cur = []
            continue
        toks = t.split()
        if len(toks) < 2:
            continue
        x, y = _parse_float(toks[0]), _parse_float(toks[1])
        if math.isnan(x) or math.isnan(y):
            continue
        if float(x).is_integer() and float(y).is_integer() and x > 1 and y > 1:
            continue  # "103. 103." point-count header
        cur.append((x, y))
    if cur:
        blocks.append(cur)
    return blocks


def parse_dat(text: str):
    """Returns (upper TE->LE, lower LE->TE, format)."""
    blocks = extract_blocks(text)
    if not blocks:
        raise ValueError("No numeric data found in DAT file.")
    first_x = blocks[0][0][0]
    if len(blocks) >= 2 and first_x < 0.1:
        return list(reversed(blocks[0])), list(blocks[1]), "lednicer"
    pts = [p for b in blocks for p in b]
    if len(pts) < 4:
        raise ValueError("Too few coordinate pairs found in DAT file.")
    le = 0
    for i in range(1, len(pts)):
        if pts[i][0] < pts[le][0]:
            le = i
    return pts[: le + 1], pts[le:], "selig"


def _catmull_rom(p0, p1, p2, p3, u):
    def knot(a, b):
        dx, dy = b[0] - a[0], b[1] - a[1]
        return math.pow(dx * dx + dy * dy, 0.25)  # centripetal, alpha = 0.5

    t0 = 0.0
    t1 = t0 + knot(p0, p1)
    t2 = t1 + knot(p1, p2)
    t3 = t2 + knot(p2, p3)
    t = t1 + u * (t2 - t1)

    def lerp(a, b, ta, tb):
        if abs(tb - ta) < 1e-12:
            return ((a[0] + b[0]) / 2, (a[1] + b[1]) / 2)
        f = (t - ta) / (tb - ta)
        return (a[0] + f * (b[0] - a[0]), a[1] + f * (b[1] - a[1]))

    A1, A2, A3 = lerp(p0, p1, t0, t1), lerp(p1, p2, t1, t2), lerp(p2, p3, t2, t3)
    B1, B2 = lerp(A1, A2, t0, t2), lerp(A2, A3, t1, t3)
    return lerp(B1, B2, t1, t2)


def build_spline(pts):
    n = len(pts)
    ph0 = (2 * pts[0][0] - pts[1][0], 2 * pts[0][1] - pts[1][1])
    phn = (2 * pts[n - 1][0] - pts[n - 2][0], 2 * pts[n - 1][1] - pts[n - 2][1])
    cp = [ph0, *pts, phn]
    al = [0.0]
    for i in range(1, n):
        dx, dy = pts[i][0] - pts[i - 1][0], pts[i][1] - pts[i - 1][1]
        al.append(al[-1] + math.sqrt(dx * dx + dy * dy))
    total = al[-1]
    tn = [v / total for v in al]

    def sample(t):
        t = max(0.0, min(1.0, t))
        lo, hi = 0, len(tn) - 2
        while lo < hi:
            mid = (lo + hi) >> 1
            if tn[mid + 1] < t:
                lo = mid + 1
            else:
                hi = mid
        seg = lo
        t0s, t1s = tn[seg], tn[seg + 1]
        u = (t - t0s) / (t1s - t0s) if t1s > t0s else 0.0
        i1 = seg + 1
        return _catmull_rom(cp[i1 - 1], cp[i1], cp[i1 + 1], cp[i1 + 2], u)

    return sample


def parse_airfoil(text: str):
    upper, lower, _ = parse_dat(text)
    lu, fl = upper[-1], lower[0]
    dup = abs(lu[0] - fl[0]) < 1e-9 and abs(lu[1] - fl[1]) < 1e-9
    contour = upper + (lower[1:] if dup else lower)
    return build_spline(contour)


def sample_airfoil(text: str, n: int, scale: float = 1.0, x_offset: float = 0.0) -> np.ndarray:
    """n body points CCW from the upper trailing edge, chord 2*scale centred at x_offset."""
    scale *= 2.0
    sample = parse_airfoil(text)
    out = np.zeros((n, 2))
    a = 5
    for k in range(n):
        x = k / n
        b = ((a - 1) * x + 0.5) / a
        s = 0.5 + math.log(b / (1 - b)) / (2 * math.log(2 * a - 1))
        px, py = sample(s)
        out[k] = ((px - 0.5) * scale + x_offset, py * scale)
    return out


def naca4(M: int, digits: int, size: float = 0.3, x_offset: float = -0.7, closed_te: bool = True) -> np.ndarray:
    """NACA 4-digit body (grid.js:38-52) from the library's host generator."""
    xy = np.zeros((M, 2), dtype=np.float64)
    _lib.check(_lib.lib().ausm_naca4_points(M, int(digits), float(size), float(x_offset), int(closed_te),
                                            xy.ctypes.data_as(C.POINTER(C.c_double))))
    return xy


def outer(M: int, kind: str = "rect", p0: float = 1.5, p1: float = 0.0, p2: float = 0.0) -> np.ndarray:
    xy = np.zeros((M, 2), dtype=np.float64)
    _lib.check(_lib.lib().ausm_outer_points(M, _lib.OUTER[kind], float(p0), float(p1), float(p2),
                                            xy.ctypes.data_as(C.POINTER(C.c_double))))
    return xy
