"""Python host binding of the C ABI (include/lbm_mutiwing.h) over ctypes.

``Simulation`` mirrors the reference's per-run state (module ``com_date`` plus
``mesh(1)``, main.f90:4-179) and its operations: creation = ini_mesh + init +
read_boundary, ``step`` = the offline loop body around ``evolution``
(main.f90:374-441), ``sums``/``reset_sums`` = the FORCE-reply accumulators
(solution.f90:379-385, driver.f90:260-289).

The CUDA library is required: when ``liblbm_b200.so`` is missing or cannot be
loaded every constructor raises; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblbm_b200.so")

PRECISION_FP64 = 0
PRECISION_FP32 = 1
MOTION_FILE = 1
MOTION_STREAM = 2
STEP_FIELDS = 1
STEP_ERR = 2
FLAG_NO_GRAPHS = 1
FLAG_SOLVE_STREAM = 2
FLAG_SOLVE_PANELS32 = 4
FLAG_SINGLE_STEPS = 8
FLAG_PASS_TALL_TILES = 16
FLAG_PASS_SHORT_TILES = 32

STATUS_BITS = {1: "band_overflow", 2: "cover_overflow", 4: "box_outside", 8: "pivot_clamped",
               16: "wings_coupled", 32: "coupled_noconv", 64: "motion"}

D = C.POINTER(C.c_double)
I32 = C.POINTER(C.c_int32)


class LbmConfig(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("scale", C.c_double), ("uu", C.c_double),
                ("re", C.c_double), ("ox", C.c_double), ("oy", C.c_double), ("s", C.c_double * 9),
                ("wing_count", C.c_int32), ("wing_x_origin", C.c_double),
                ("wing_x_spacing", C.c_double), ("wing_y_origin", C.c_double),
                ("xc", C.c_double), ("yc", C.c_double), ("motion_source", C.c_int32),
                ("precision", C.c_int32), ("device", C.c_int32), ("flags", C.c_int32),
                ("reserved", C.c_int32 * 6)]


# (name, restype, argtypes) of every exported entry point
SIGNATURES = [
    ("lbm_abi_version", C.c_int, []),
    ("lbm_config_default", None, [C.POINTER(LbmConfig)]),
    ("lbm_create", C.c_int, [C.POINTER(LbmConfig), D, I32, C.POINTER(C.c_void_p)]),
    ("lbm_reset", C.c_int, [C.c_void_p]),
    ("lbm_set_motion_table", C.c_int, [C.c_void_p, D, C.c_int64, C.c_int32]),
    ("lbm_set_stream_rows", C.c_int, [C.c_void_p, D, D]),
    ("lbm_build_stream_target_row", C.c_int, [C.c_void_p, D, C.c_double, D, D]),
    ("lbm_step", C.c_int, [C.c_void_p, C.c_int64, C.c_int64, D, C.c_int32]),
    ("lbm_get_sums", C.c_int, [C.c_void_p, D, I32, I32]),
    ("lbm_reset_sums", C.c_int, [C.c_void_p]),
    ("lbm_get_fields", C.c_int, [C.c_void_p, D, D, D, D]),
    ("lbm_get_output", C.c_int, [C.c_void_p, C.c_int32, C.c_int32, D, D, D, D]),
    ("lbm_err", C.c_int, [C.c_void_p, D]),
    ("lbm_err_fields_noalloc", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32,
                                         C.c_int64, C.c_int32, C.c_void_p, D, C.c_char_p, C.c_int32]),
    ("lbm_get_f", C.c_int, [C.c_void_p, D]),
    ("lbm_get_border_f0", C.c_int, [C.c_void_p, D, I32]),
    ("lbm_set_border_f0", C.c_int, [C.c_void_p, D, C.c_int32]),
    ("lbm_set_f", C.c_int, [C.c_void_p, D]),
    ("lbm_get_band", C.c_int, [C.c_void_p, I32, I32, C.c_int32]),
    ("lbm_get_markers", C.c_int, [C.c_void_p, D, D, D, D]),
    ("lbm_move_mesh", C.c_int, [C.c_void_p, C.c_int32]),
    ("lbm_ibm_residual", C.c_int, [C.c_void_p, D]),
    ("lbm_status", C.c_int, [C.c_void_p, I32]),
    ("lbm_set_timing", C.c_int, [C.c_void_p, C.c_int32]),
    ("lbm_get_phase_times", C.c_int, [C.c_void_p, D, C.c_int32]),
    ("lbm_stream", C.c_void_p, [C.c_void_p]),
    ("lbm_device_bytes", C.c_int64, [C.c_void_p]),
    ("lbm_mem_info", C.c_int, [C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    ("lbm_last_error", C.c_char_p, [C.c_void_p]),
    ("lbm_destroy", None, [C.c_void_p]),
    ("lbm_batch_create", C.c_int, [C.c_int32, C.POINTER(C.c_void_p)]),
    ("lbm_batch_step", C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_void_p), C.POINTER(C.c_int64),
                                 C.POINTER(C.c_int64), C.POINTER(D), I32, I32]),
    ("lbm_batch_last_error", C.c_char_p, [C.c_void_p]),
    ("lbm_batch_destroy", None, [C.c_void_p]),
]

_lib = None


class LbmError(RuntimeError):
    pass


def load_library(path: Optional[str] = None):
    """Load the CUDA library (``path``, else the module's ``LIB_PATH`` at the
    first call); raises if it is absent (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise LbmError(f"{path} is missing: build it with `python -m lbm_mutiwing_b200.build`")
    lib = C.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.lbm_abi_version() != 1:
        raise LbmError("ABI version mismatch")
    _lib = lib
    return lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(D)


def mem_info(device: int = 0):
    """(free, total) bytes of the device (lbm_mem_info)."""
    L = load_library()
    fr, to = C.c_int64(0), C.c_int64(0)
    if L.lbm_mem_info(device, C.byref(fr), C.byref(to)) != 0:
        raise LbmError(f"cannot query the memory of CUDA device {device}")
    return fr.value, to.value


def estimate_device_bytes(ep, precision: int) -> int:
    """Upper bound of the device memory an episode takes before it is
    created: per node the distributions (FP32 path: two copies of nine FP32
    planes; FP64 path: f and f0 in FP64 and eight FP64 fields), the band maps
    and bit planes, and the fields written on request (FP32 path), plus a
    fixed 64 MB for the immersed-boundary arrays, force rows and graphs."""
    per_node = 120 if precision == PRECISION_FP32 else 212
    return per_node * ep.nx * ep.ny + (64 << 20)


def default_s() -> list:
    """MRT rates of ini_mesh.f90:59-67 (the two stress rates default to 1/tau)."""
    return [0.0, 1.1, 1.05, 0.0, 1.2, 0.0, 1.2, 0.0, 0.0]


def make_config(ep, precision: int = PRECISION_FP64, motion_source: int = MOTION_FILE,
                device: int = 0, s: Optional[Sequence[float]] = None, graphs: bool = True,
                flags: int = 0) -> LbmConfig:
    cfg = LbmConfig()
    cfg.flags = (0 if graphs else FLAG_NO_GRAPHS) | flags
    cfg.nx, cfg.ny = ep.nx, ep.ny
    cfg.scale, cfg.uu, cfg.re = ep.scale, ep.uu, ep.re
    cfg.ox, cfg.oy = ep.ox, ep.oy
    for k, v in enumerate(s if s is not None else default_s()):
        cfg.s[k] = v
    cfg.wing_count = ep.wing_count
    cfg.wing_x_origin, cfg.wing_x_spacing, cfg.wing_y_origin = (
        ep.wing_x_origin, ep.wing_x_spacing, ep.wing_y_origin)
    cfg.xc = cfg.yc = 0.0
    cfg.motion_source = motion_source
    cfg.precision = precision
    cfg.device = device
    return cfg


class Simulation:
    """One episode resident on one GPU."""

    def __init__(self, ep, precision: int = PRECISION_FP64, motion_source: int = MOTION_FILE,
                 device: int = 0, s: Optional[Sequence[float]] = None, load_motion: bool = True,
                 graphs: bool = True, flags: int = 0):
        self.L = load_library()
        self.ep = ep
        self.cfg = make_config(ep, precision, motion_source, device, s, graphs, flags)
        self.nx, self.ny, self.W = ep.nx, ep.ny, ep.wing_count
        self.precision = precision
        self.row_len = 4 + 12 * self.W
        xy = np.ascontiguousarray(ep.markers_xy().reshape(-1), dtype=np.float64)
        ppw = np.ascontiguousarray(ep.points_per_wing(), dtype=np.int32)
        self.npts = int(ppw.sum())
        self.nseg = int((ppw - 1).sum())
        h = C.c_void_p()
        rc = self.L.lbm_create(C.byref(self.cfg), _dp(xy) if xy.size else None,
                               ppw.ctypes.data_as(I32) if ppw.size else None, C.byref(h))
        self.h = h
        if rc != 0:
            msg = self.L.lbm_last_error(h).decode() if h.value else "lbm_create failed"
            if h.value:
                self.L.lbm_destroy(h)
            self.h = None
            raise LbmError(msg)
        self.cycle = 1
        if load_motion and ep.motion is not None and motion_source == MOTION_FILE:
            self.set_motion_table(ep.motion)

    # -- lifecycle
    def close(self):
        if getattr(self, "h", None):
            self.L.lbm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc: int):
        if rc != 0:
            raise LbmError(self.L.lbm_last_error(self.h).decode())

    # -- operations
    def reset(self):
        self._check(self.L.lbm_reset(self.h))
        self.cycle = 1

    def set_motion_table(self, rows):
        rows = np.ascontiguousarray(rows, dtype=np.float64)
        self._check(self.L.lbm_set_motion_table(self.h, _dp(rows), rows.shape[0], rows.shape[1]))

    def set_stream_rows(self, start, target):
        a = np.ascontiguousarray(start, dtype=np.float64)
        b = np.ascontiguousarray(target, dtype=np.float64)
        self._check(self.L.lbm_set_stream_rows(self.h, _dp(a), _dp(b)))

    def build_stream_target_row(self, start, target_time, delta):
        a = np.ascontiguousarray(start, dtype=np.float64)
        d = np.ascontiguousarray(delta, dtype=np.float64)
        out = np.zeros(1 + 9 * self.W)
        rc = self.L.lbm_build_stream_target_row(self.h, _dp(a), target_time, _dp(d), _dp(out))
        if rc != 0:
            raise LbmError("STEP time must not precede the segment start")
        return out

    def step(self, n_steps: int = 1, first_cycle: Optional[int] = None, rows: bool = True,
             flags: int = 0) -> Optional[np.ndarray]:
        """Advance n_steps cycles; returns the force rows (n_steps x (4+12W))."""
        first = self.cycle if first_cycle is None else first_cycle
        out = np.zeros((n_steps, self.row_len)) if rows else None
        self._check(self.L.lbm_step(self.h, first, n_steps, _dp(out) if rows and n_steps else None, flags))
        self.cycle = first + n_steps
        return out

    def sums(self):
        s = np.zeros(self.row_len)
        cnt, ln = C.c_int32(0), C.c_int32(0)
        self._check(self.L.lbm_get_sums(self.h, _dp(s), C.byref(cnt), C.byref(ln)))
        return s, cnt.value, ln.value

    def reset_sums(self):
        self._check(self.L.lbm_reset_sums(self.h))

    def fields(self):
        """rho, u, v, pre as (ny, nx) arrays."""
        arrs = [np.zeros((self.ny, self.nx)) for _ in range(4)]
        self._check(self.L.lbm_get_fields(self.h, *[_dp(a) for a in arrs]))
        return tuple(arrs)

    def output(self, stride_x: int = 2, stride_y: int = 2):
        """u/UU, v/UU, pre, vorticity at the output nodes as (ony, onx) arrays
        (output, solution.f90:132-241)."""
        onx, ony = (self.nx - 1) // stride_x + 1, (self.ny - 1) // stride_y + 1
        arrs = [np.zeros((ony, onx)) for _ in range(4)]
        self._check(self.L.lbm_get_output(self.h, stride_x, stride_y, *[_dp(a) for a in arrs]))
        return tuple(arrs)

    def err(self) -> float:
        e = C.c_double()
        self._check(self.L.lbm_err(self.h, C.byref(e)))
        return e.value

    def f(self) -> np.ndarray:
        out = np.zeros((9, self.ny, self.nx))
        self._check(self.L.lbm_get_f(self.h, _dp(out)))
        return out

    def set_f(self, f):
        a = np.ascontiguousarray(f, dtype=np.float64)
        self._check(self.L.lbm_set_f(self.h, _dp(a)))

    def border_f0(self):
        """(f0 of the border nodes, 9 x (2 ny + 2 nx); movenum)."""
        out = np.zeros((9, 2 * self.ny + 2 * self.nx))
        m = C.c_int32(0)
        self._check(self.L.lbm_get_border_f0(self.h, _dp(out), C.byref(m)))
        return out, m.value

    def set_border_f0(self, f0, movenum: int):
        a = np.ascontiguousarray(f0, dtype=np.float64)
        if a.size != 9 * (2 * self.ny + 2 * self.nx):
            raise LbmError("border f0 must hold 9 x (2 ny + 2 nx) values")
        self._check(self.L.lbm_set_border_f0(self.h, _dp(a), int(movenum)))

    def band(self) -> np.ndarray:
        n = C.c_int32(0)
        self._check(self.L.lbm_get_band(self.h, C.byref(n), None, 0))
        out = np.zeros(3 * max(n.value, 1), dtype=np.int32)
        self._check(self.L.lbm_get_band(self.h, C.byref(n), out.ctypes.data_as(I32), n.value))
        return out[:3 * n.value].reshape(-1, 3)

    def markers(self):
        xb1, yb1 = np.zeros(self.npts), np.zeros(self.npts)
        xb2, yb2 = np.zeros(self.nseg), np.zeros(self.nseg)
        self._check(self.L.lbm_get_markers(self.h, _dp(xb1), _dp(yb1), _dp(xb2), _dp(yb2)))
        return xb1, yb1, xb2, yb2

    def move_mesh(self, dr: int):
        self._check(self.L.lbm_move_mesh(self.h, dr))

    def ibm_residual(self) -> float:
        r = C.c_double()
        self._check(self.L.lbm_ibm_residual(self.h, C.byref(r)))
        return r.value

    def status(self) -> int:
        b = C.c_int32()
        self._check(self.L.lbm_status(self.h, C.byref(b)))
        return b.value

    def set_timing(self, enable: bool = True):
        self._check(self.L.lbm_set_timing(self.h, 1 if enable else 0))

    def phase_times(self) -> dict:
        out = np.zeros(10)
        self._check(self.L.lbm_get_phase_times(self.h, _dp(out), 10))
        return {"move_boundary_ms": out[0], "collide_stream_ms": out[1], "band_ms": out[2],
                "bc_ms": out[3], "ibm_solve_ms": out[4], "ibm_factor_ms": out[5], "steps": int(out[6]),
                "pass_far_ms": out[7], "passes": int(out[8]), "far_tile_nodes": int(out[9])}

    def stream(self) -> int:
        return int(self.L.lbm_stream(self.h) or 0)

    def device_bytes(self) -> int:
        return int(self.L.lbm_device_bytes(self.h))


class BatchStepError(LbmError):
    """Raised by Batch.step when episodes failed; rcs[i] != 0 marks them and
    messages[i] holds each failed episode's error text.  When some rcs are
    non-zero the call did step every episode (an episode fails its status
    check after the steps): outs[i] holds the force rows of the others, and
    every episode's cycle has advanced with its device state."""

    def __init__(self, msg, rcs, messages, outs=None):
        super().__init__(msg)
        self.rcs = rcs
        self.messages = messages
        self.outs = outs if outs is not None else [None] * len(rcs)


class Batch:
    """Packed stepping of many FP32-path episodes on one device
    (lbm_batch_step): each step is one launch per kernel over every episode
    still stepping, with results identical to stepping each episode alone."""

    def __init__(self, device: int = 0):
        self.L = load_library()
        h = C.c_void_p()
        rc = self.L.lbm_batch_create(device, C.byref(h))
        self.h = h
        if rc != 0:
            msg = self.L.lbm_batch_last_error(h).decode() if h.value else "lbm_batch_create failed"
            if h.value:
                self.L.lbm_batch_destroy(h)
            self.h = None
            raise LbmError(msg)

    def close(self):
        if getattr(self, "h", None):
            self.L.lbm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def step(self, sims: Sequence["Simulation"], n_steps, first_cycles=None, rows: bool = True, flags=0):
        """Advance sims[i] by n_steps[i] (an int applies to all) from
        first_cycles[i] (default: each simulation's next cycle); returns the
        force rows of each (None where rows is False)."""
        n = len(sims)
        if n == 0:
            return []
        ns = [int(n_steps)] * n if np.isscalar(n_steps) else [int(x) for x in n_steps]
        fl = [int(flags)] * n if np.isscalar(flags) else [int(x) for x in flags]
        first = [s.cycle for s in sims] if first_cycles is None else [int(x) for x in first_cycles]
        outs = [np.zeros((k, s.row_len)) if rows and k else None for s, k in zip(sims, ns)]
        hs = (C.c_void_p * n)(*[s.h.value for s in sims])
        fc = (C.c_int64 * n)(*first)
        nn = (C.c_int64 * n)(*ns)
        rp = (D * n)(*[_dp(o) if o is not None else D() for o in outs])
        ff = (C.c_int32 * n)(*fl)
        rcs = (C.c_int32 * n)()
        rc = self.L.lbm_batch_step(self.h, n, hs, fc, nn, rp, ff, rcs)
        if rc != 0:
            codes = list(rcs)
            msgs = [sims[i].L.lbm_last_error(sims[i].h).decode() if codes[i] else "" for i in range(n)]
            stepped = any(codes)
            if stepped:
                # every episode was stepped (the failed ones failed their
                # status check afterwards): host cycles follow the device
                for s, f0, k in zip(sims, first, ns):
                    s.cycle = f0 + k
            raise BatchStepError(self.L.lbm_batch_last_error(self.h).decode(), codes, msgs,
                                 [o if stepped and not c else None for o, c in zip(outs, codes)])
        for s, f0, k in zip(sims, first, ns):
            s.cycle = f0 + k
        return outs


def finalize_force_average(sum_row: np.ndarray, count: int, row_len: int, wing_count: int,
                           end_time: float, last_row: np.ndarray) -> np.ndarray:
    """finalize_force_reply_average (driver.f90:270-289): average the force
    columns 2 .. 1+3W+3 over the segment, keep the last step's motion columns
    and set column 1 to the segment end time."""
    if count <= 0:
        return np.zeros(0)
    out = np.array(last_row[:row_len], dtype=np.float64, copy=True)
    end = min(row_len, 1 + 3 * wing_count + 3)
    out[1:end] = sum_row[1:end] / float(count)
    out[0] = end_time
    return out
