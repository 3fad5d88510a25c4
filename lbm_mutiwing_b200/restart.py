"""Restart files in the reference's layout (saveflowfield / readflowfield,
solution.f90:1616-1851): `saved_flow_feild.dat` and its copy
`saved_flow_feild_copy.dat`, written with `form='binary'` (a raw stream, no
record markers; default 4-byte integers, 8-byte reals, little-endian):

    int32  cycle1
    int32  wing_count
    float64 x 11 W   body_rel_a, _a_prev, _v, _v_prev, _s, _s_prev, _pos,
                     _theta_prev, _theta, _temp_theta_prev, _temp_theta
    int32  movenum
    for j = 1..Ny, i = 1..Nx:       u(i,j), v(i,j), f(i,j,1:9)
    for j = 2..Ny-1:                leftf2(j,:), f0(1,j,:), rightf2(j,:), f0(Nx,j,:)
    for i = 1..Nx:                  upf2(i,:), f0(i,Ny,:), downf2(i,:), f0(i,1,:)

leftf2 / rightf2 / upf2 / downf2 keep the border populations of set-up
(solution.f90:60-63); on this path nothing updates them afterwards
(boundary_condition1 does not), so they are the initial equilibrium
feq(1, UU, 0).  The rigid-body relative motion is zero unless the dynamics
solver is enabled, which this path does not support: a file with non-zero
relative motion is refused.
"""
from __future__ import annotations

import os
from typing import Tuple

import numpy as np

FILE = "saved_flow_feild.dat"
COPY = "saved_flow_feild_copy.dat"

# D2Q9 weights as the reference's single-precision literals (D2Q9model.f90)
_W = np.array([4.0 / 9.0] + [1.0 / 9.0] * 4 + [1.0 / 36.0] * 4, dtype=np.float32).astype(np.float64)
_EX = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1], dtype=np.float64)
_EY = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1], dtype=np.float64)


def initial_equilibrium(uu: float) -> np.ndarray:
    """feq(rho = 1, u = UU, v = 0) (D2Q9feq, D2Q9model.f90:30-46)."""
    eu = _EX * uu
    return _W * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * uu * uu)


def _border_layout(nx: int, ny: int):
    """Index of each border node in the library's border f0 vector (left
    column, right column, bottom row, top row)."""
    left = np.arange(ny)
    right = ny + np.arange(ny)
    bottom = 2 * ny + np.arange(nx)
    top = 2 * ny + nx + np.arange(nx)
    return left, right, bottom, top


def encode(cycle: int, wing_count: int, movenum: int, u: np.ndarray, v: np.ndarray, f: np.ndarray,
           border_f0: np.ndarray, uu: float) -> bytes:
    """The file's bytes.  u, v: (ny, nx); f: (9, ny, nx); border_f0: (9, 2 ny + 2 nx)."""
    ny, nx = u.shape
    head = np.array([cycle, wing_count], dtype="<i4").tobytes()
    rel = np.zeros(11 * wing_count, dtype="<f8").tobytes()
    mv = np.array([movenum], dtype="<i4").tobytes()
    nodes = np.empty((ny, nx, 11), dtype="<f8")
    nodes[:, :, 0] = u
    nodes[:, :, 1] = v
    nodes[:, :, 2:] = np.moveaxis(f, 0, -1)
    feq = initial_equilibrium(uu)
    left, right, bottom, top = _border_layout(nx, ny)
    cols = np.empty((ny - 2, 4, 9), dtype="<f8")
    cols[:, 0] = feq
    cols[:, 1] = border_f0[:, left[1:ny - 1]].T
    cols[:, 2] = feq
    cols[:, 3] = border_f0[:, right[1:ny - 1]].T
    rows = np.empty((nx, 4, 9), dtype="<f8")
    rows[:, 0] = feq
    rows[:, 1] = border_f0[:, top].T
    rows[:, 2] = feq
    rows[:, 3] = border_f0[:, bottom].T
    return head + rel + mv + nodes.tobytes() + cols.tobytes() + rows.tobytes()


def decode(data: bytes, nx: int, ny: int, wing_count: int):
    """(cycle, movenum, u, v, f, border_f0) from a file's bytes; the border
    columns' f0 of rows 1 and ny come from the row records, as the reader
    overwrites them in that order (solution.f90:1765-1776)."""
    want = 12 + 88 * wing_count + 88 * nx * ny + 288 * (ny - 2) + 288 * nx
    if len(data) != want:
        raise ValueError(f"restart file has {len(data)} bytes, expected {want} for {nx} x {ny} and {wing_count} wings")
    cycle, wc = np.frombuffer(data, "<i4", 2, 0)
    if wc != wing_count:
        raise ValueError(f"restart file holds {wc} wings, the episode has {wing_count}")
    o = 8
    rel = np.frombuffer(data, "<f8", 11 * wing_count, o)
    o += 88 * wing_count
    if np.any(rel != 0.0):
        raise ValueError("restart file carries rigid-body relative motion, which this path does not support")
    movenum = int(np.frombuffer(data, "<i4", 1, o)[0])
    o += 4
    nodes = np.frombuffer(data, "<f8", 11 * nx * ny, o).reshape(ny, nx, 11)
    o += 88 * nx * ny
    cols = np.frombuffer(data, "<f8", 36 * (ny - 2), o).reshape(ny - 2, 4, 9)
    o += 288 * (ny - 2)
    rows = np.frombuffer(data, "<f8", 36 * nx, o).reshape(nx, 4, 9)
    u = nodes[:, :, 0].copy()
    v = nodes[:, :, 1].copy()
    f = np.ascontiguousarray(np.moveaxis(nodes[:, :, 2:], -1, 0))
    border = np.zeros((9, 2 * ny + 2 * nx))
    left, right, bottom, top = _border_layout(nx, ny)
    border[:, left[1:ny - 1]] = cols[:, 1].T
    border[:, right[1:ny - 1]] = cols[:, 3].T
    border[:, top] = rows[:, 1].T
    border[:, bottom] = rows[:, 3].T
    # the corner columns' f0 at rows 1 and ny: the row records (i = 1, Nx)
    border[:, left[0]] = rows[0, 3]
    border[:, left[ny - 1]] = rows[0, 1]
    border[:, right[0]] = rows[nx - 1, 3]
    border[:, right[ny - 1]] = rows[nx - 1, 1]
    return int(cycle), movenum, u, v, f, border


def save(out_dir: str, sim, cycle: int) -> Tuple[str, str]:
    """saveflowfield: both files, after a step that wrote the fields
    (lbm_step with LBM_STEP_FIELDS, or any plain-path step)."""
    _, u, v, _ = sim.fields()
    f = sim.f()
    border, movenum = sim.border_f0()
    data = encode(cycle, sim.W, movenum, u, v, f, border, sim.ep.uu)
    os.makedirs(out_dir, exist_ok=True)
    paths = (os.path.join(out_dir, FILE), os.path.join(out_dir, COPY))
    for p in paths:
        with open(p, "wb") as fh:
            fh.write(data)
    return paths


def load(in_dir: str, sim) -> int:
    """readflowfield: the first readable file (the copy when the main file
    is missing or short); sets the distributions, the border f0 and movenum;
    returns the cycle the run continues from."""
    last = None
    for name in (FILE, COPY):
        p = os.path.join(in_dir, name)
        try:
            with open(p, "rb") as fh:
                data = fh.read()
            cycle, movenum, _, _, f, border = decode(data, sim.nx, sim.ny, sim.W)
        except (OSError, ValueError) as e:
            last = e
            if isinstance(e, ValueError) and "wings" in str(e):
                raise
            continue
        sim.set_f(f)
        sim.set_border_f0(border, movenum)
        sim.cycle = cycle
        return cycle
    raise ValueError(f"no readable restart file in {in_dir}: {last}")
