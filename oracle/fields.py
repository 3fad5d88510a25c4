"""Field comparisons against the oracle -- TEST INFRASTRUCTURE ONLY.

Loaded by tests/ and by the benchmark's CPU-baseline leg (which runs the
oracle once and both times it and compares the GPU paths with it), never by
the product package.

* ``vorticity`` restates the vorticity of the reference's ``output``
  (solution.f90:185-205): dv/dx - du/dy in units of UU/scale, centred
  differences inside, second-order one-sided differences on the border rows
  and columns, evaluated on every node (stride 1).
* ``field_errors`` gives the relative L2 errors of u, v, p and vorticity
  (||a - b|| / ||b|| over all nodes).
* ``segment_average`` and ``force_error`` give the segment-averaged per-wing
  Fx, Fy, M of a block of force rows (the FORCE reply average of
  driver.f90:260-289: columns 2 .. 1+3W of the force-row layout of
  solution.f90:352-378) and the largest relative error of one average against
  another, relative per quantity to the largest magnitude of that quantity
  over the wings.
"""
from __future__ import annotations

import numpy as np


def vorticity(u: np.ndarray, v: np.ndarray, uu: float, scale: float) -> np.ndarray:
    """dv/dx - du/dy on an (ny, nx) lattice, solution.f90:185-205."""
    ny, nx = u.shape
    dvx = np.empty_like(v)
    dvx[:, 1:-1] = (v[:, 2:] - v[:, :-2]) / (uu * 2.0 * scale)
    dvx[:, -1] = (1.5 * v[:, -1] - 2.0 * v[:, -2] + 0.5 * v[:, -3]) / (uu * scale)
    dvx[:, 0] = (-1.5 * v[:, 0] + 2.0 * v[:, 1] - 0.5 * v[:, 2]) / (uu * scale)
    duy = np.empty_like(u)
    duy[1:-1, :] = (u[2:, :] - u[:-2, :]) / (uu * 2.0 * scale)
    duy[-1, :] = (1.5 * u[-1, :] - 2.0 * u[-2, :] + 0.5 * u[-3, :]) / (uu * scale)
    duy[0, :] = (-1.5 * u[0, :] + 2.0 * u[1, :] - 0.5 * u[2, :]) / (uu * scale)
    return dvx - duy


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.linalg.norm(a - b) / max(float(np.linalg.norm(b)), 1e-300))


def field_errors(u, v, p, u_ref, v_ref, p_ref, uu: float, scale: float) -> dict:
    """Relative L2 errors of u, v, p and vorticity against reference fields."""
    return {"u_l2": rel_l2(u, u_ref), "v_l2": rel_l2(v, v_ref), "p_l2": rel_l2(p, p_ref),
            "vort_l2": rel_l2(vorticity(u, v, uu, scale), vorticity(u_ref, v_ref, uu, scale))}


def segment_average(rows: np.ndarray, wing_count: int) -> np.ndarray:
    """(wing_count, 3) mean per-wing Fx, Fy, M over the rows."""
    return rows[:, 1:1 + 3 * wing_count].mean(axis=0).reshape(wing_count, 3)


def force_error(avg: np.ndarray, ref: np.ndarray) -> float:
    """Largest |avg - ref| over wings and quantities, each quantity scaled by
    its largest |ref| over the wings."""
    scale = np.maximum(np.abs(ref).max(axis=0), 1e-300)
    return float((np.abs(avg - ref) / scale).max())
