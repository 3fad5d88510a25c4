"""Output files of a run, in the reference's text formats.

* ``write_flow_field`` -- the Tecplot file ``F<cycle>.dat`` of ``output``
  (solution.f90:132-241): a structured zone of the strided lattice with X, Y,
  U, V, pressure, vorticity, body and dvordt (format 25e16.8), then the
  airfoil as a finite-element zone (markers, one centre node per wing,
  triangles of each segment with its wing's centre).  The field values come
  from ``lbm_get_output`` (computed on the device); ``body`` and ``dvordt``
  are zero, as in the reference, whose vorticity-rate routine is disabled
  (main.f90:414).
* ``ForceWriter`` -- the per-step ``force*.dat`` and ``airfoil_motion*.dat``
  rows of evolution (solution.f90:386-402), format 1000f15.8.

Fortran edit descriptors are restated here (E, F, I); the list-directed
ZONE header lines follow gfortran's list-directed layout.
"""
from __future__ import annotations

import math
import os
from typing import Sequence

import numpy as np


def fortran_e(x: float, w: int = 16, d: int = 8) -> str:
    """Fortran Ew.d: optional sign, '0.', d digits, exponent E+dd (or +ddd
    when the exponent needs three digits), right-justified in w."""
    if math.isnan(x):
        return "NaN".rjust(w)
    if math.isinf(x):
        return ("-Infinity" if x < 0 else "Infinity").rjust(w)
    neg = math.copysign(1.0, x) < 0
    a = abs(x)
    if a == 0.0:
        mant, exp = "0" * d, 0
    else:
        s = f"{a:.{d - 1}E}"          # d significant digits, 1 <= m < 10
        m, e = s.split("E")
        mant, exp = m.replace(".", ""), int(e) + 1
    ex = f"E{'-' if exp < 0 else '+'}{abs(exp):02d}" if abs(exp) <= 99 else f"{'-' if exp < 0 else '+'}{abs(exp):03d}"
    out = ("-" if neg else "") + "0." + mant + ex
    return out.rjust(w)


def fortran_f(x: float, w: int, d: int) -> str:
    """Fortran Fw.d (asterisks when the value does not fit)."""
    s = f"{x:{w}.{d}f}"
    return s if len(s) <= w else "*" * w


def fortran_i(k: int, w: int, m: int = 1) -> str:
    """Fortran Iw.m: at least m digits, right-justified in w."""
    s = ("-" if k < 0 else "") + str(abs(k)).rjust(m, "0")
    return s.rjust(w) if len(s) <= w else "*" * w


def _list_int(k: int) -> str:
    return str(k).rjust(12)


def _list_real(x: float) -> str:
    m, e = f"{x:.16E}".split("E")
    return (m + "E" + e[0] + e[1:].rjust(3, "0")).rjust(25)


def format_row_1000f15_8(values: Sequence[float]) -> str:
    return "".join(fortran_f(float(v), 15, 8) for v in values)


def write_flow_field(path: str, cycle: int, ep, u: np.ndarray, v: np.ndarray, pre: np.ndarray,
                     vort: np.ndarray, stride_x: int, stride_y: int, xb1: np.ndarray, yb1: np.ndarray,
                     points_per_wing: Sequence[int], movenum: int = 0) -> None:
    """The Tecplot file of output (solution.f90:165-236) for one episode.
    u, v, pre, vort: (ony, onx) arrays from ``Simulation.output``; xb1, yb1 the
    current markers of all wings back to back."""
    ony, onx = u.shape
    scale, uu = ep.scale, ep.uu
    t = cycle * uu * scale
    lines = ['VARIABLES = "X" "Y" "U" "V" "Presure" "Vorticity" "body" "dvordt" ',
             ' ZONE T="Flow feild", I=' + _list_int(onx) + ' ,J=' + _list_int(ony) +
             ' ,SOLUTIONTIME=' + _list_real(t)]
    xs = ep.ox + np.arange(0, ep.nx, stride_x, dtype=np.float64) * scale + movenum * scale
    ys = ep.oy + np.arange(0, ep.ny, stride_y, dtype=np.float64) * scale
    for oj in range(ony):
        y = ys[oj]
        for oi in range(onx):
            lines.append("".join(fortran_e(val) for val in
                                 (xs[oi], y, u[oj, oi], v[oj, oi], pre[oj, oi], vort[oj, oi], 0.0, 0.0)))
    b_point = int(sum(points_per_wing))
    nseg = int(sum(n - 1 for n in points_per_wing))
    W = len(points_per_wing)
    lines.append(' ZONE T="airfoil", NODES=' + _list_int(b_point + W) + ' ELEMENTS,=' + _list_int(nseg) +
                 ', DATAPACKING=POINT, ZONETYPE=FETRIANGLE' + ',SOLUTIONTIME=' + _list_real(t))
    def node(x, y):
        return "".join(fortran_f(val, 14, 8) for val in (x, y, 255.0, 0.0, 0.0, 0.0, 0.0, 0.0))
    for p in range(b_point):
        lines.append(node(xb1[p] + movenum * scale, yb1[p]))
    start = 0
    starts = []
    for n in points_per_wing:
        starts.append(start)
        start += n
    for w in range(W):
        j = starts[w]
        k = j + (points_per_wing[w] - 1) // 2
        lines.append(node(0.5 * ((xb1[j] + movenum * scale) + (xb1[k] + movenum * scale)), 0.5 * (yb1[j] + yb1[k])))
    for w in range(W):
        j = starts[w] + 1                    # 1-based point numbers
        for k in range(j, j + points_per_wing[w] - 1):
            lines.append(fortran_i(k, 5, 3) + fortran_i(k + 1, 5, 3) + fortran_i(b_point + w + 1, 5, 3))
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


class ForceWriter:
    """force_episode_<k>.dat and airfoil_motion_episode_<k>.dat
    (driver.f90:410-428) with one row per step (solution.f90:386-402)."""

    def __init__(self, out_dir: str, episode: int, wing_count: int, x_origin: float, x_spacing: float):
        os.makedirs(out_dir, exist_ok=True)
        self.W = wing_count
        self.f = open(os.path.join(out_dir, f"force_episode_{episode}.dat"), "w")
        self.m = open(os.path.join(out_dir, f"airfoil_motion_episode_{episode}.dat"), "w")

    def add(self, rows: np.ndarray) -> None:
        """rows: force rows (n x (4 + 12W)) of consecutive steps."""
        W = self.W
        for r in rows:
            self.f.write(format_row_1000f15_8(r) + "\n")
            mot = [r[0]]
            for w in range(W):
                x_abs = r[4 + 3 * W + 9 * w]     # absolute x of the wing (solution.f90:366-367)
                mot += [0.0, 0.0, x_abs]         # extra_v is zero without body dynamics
            self.m.write(format_row_1000f15_8(mot) + "\n")
        self.f.flush()
        self.m.flush()

    def close(self) -> None:
        for fh in (self.f, self.m):
            if not fh.closed:
                fh.close()
