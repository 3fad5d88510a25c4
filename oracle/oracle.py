"""ctypes binding for the CPU FP64 oracle (test infrastructure only).

Imported by tests/, by ``__graft_entry__.smoke()`` and by the benchmark's
CPU-baseline leg, never by the product package.  ``build()`` compiles the
library with oracle/Makefile.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblbm_oracle.so")

D = C.POINTER(C.c_double)
I = C.POINTER(C.c_int32)


class OraConfig(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("scale", C.c_double), ("uu", C.c_double),
                ("re", C.c_double), ("ox", C.c_double), ("oy", C.c_double), ("s", C.c_double * 9),
                ("wing_count", C.c_int32), ("wing_x_origin", C.c_double),
                ("wing_x_spacing", C.c_double), ("wing_y_origin", C.c_double),
                ("xc", C.c_double), ("yc", C.c_double), ("motion_source", C.c_int32)]


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "lbm_oracle.cpp")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE, "liblbm_oracle.so"], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.ora_create.restype = C.c_void_p
        L.ora_create.argtypes = [C.POINTER(OraConfig), D, I, C.c_int32]
        L.ora_destroy.argtypes = [C.c_void_p]
        L.ora_set_motion_table.argtypes = [C.c_void_p, D, C.c_int64, C.c_int32]
        L.ora_set_stream_rows.argtypes = [C.c_void_p, D, D]
        L.ora_step.argtypes = [C.c_void_p, C.c_int64, D]
        L.ora_err.restype = C.c_double
        L.ora_err.argtypes = [C.c_void_p]
        L.ora_tau.restype = C.c_double
        L.ora_tau.argtypes = [C.c_void_p]
        L.ora_get_field.argtypes = [C.c_void_p, C.c_int32, D]
        L.ora_set_f.argtypes = [C.c_void_p, D]
        L.ora_get_band.argtypes = [C.c_void_p, I, I, C.c_int32]
        L.ora_get_markers.argtypes = [C.c_void_p, D, D, D, D]
        L.ora_get_sums.argtypes = [C.c_void_p, D, I, I]
        L.ora_reset_sums.argtypes = [C.c_void_p]
        L.ora_stream_row.argtypes = [C.c_void_p, C.c_double, D]
        L.ora_build_stream_target_row.argtypes = [C.c_void_p, D, C.c_double, D, D]
        L.ora_interpolate_triplet.argtypes = [C.c_double] * 5 + [D, D, D]
        L.ora_delta_phi.restype = C.c_double
        L.ora_delta_phi.argtypes = [C.c_double]
        L.ora_inverse_m.argtypes = [D]
        L.ora_move_mesh.argtypes = [C.c_void_p, C.c_int32]
        L.ora_ibm_residual.restype = C.c_double
        L.ora_ibm_residual.argtypes = [C.c_void_p]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(D)


def default_s():
    """MRT rates of ini_mesh.f90:59-67; the two stress rates (<= 0) become 1/tau."""
    return [0.0, 1.1, 1.05, 0.0, 1.2, 0.0, 1.2, 0.0, 0.0]


class Oracle:
    """One simulation held by the oracle; mirrors the reference's global state."""

    def __init__(self, ep, nthreads: int = 1, motion_source: int = 1, s=None):
        self.L = lib()
        cfg = OraConfig()
        cfg.nx, cfg.ny, cfg.scale, cfg.uu, cfg.re = ep.nx, ep.ny, ep.scale, ep.uu, ep.re
        cfg.ox, cfg.oy = ep.ox, ep.oy
        for k, v in enumerate(s if s is not None else default_s()):
            cfg.s[k] = v
        cfg.wing_count = ep.wing_count
        cfg.wing_x_origin, cfg.wing_x_spacing, cfg.wing_y_origin = (
            ep.wing_x_origin, ep.wing_x_spacing, ep.wing_y_origin)
        cfg.xc = cfg.yc = 0.0
        cfg.motion_source = motion_source
        self.nx, self.ny, self.W = ep.nx, ep.ny, ep.wing_count
        xy = ep.markers_xy()
        self._xy = np.ascontiguousarray(xy.reshape(-1), dtype=np.float64)
        self._ppw = np.ascontiguousarray(ep.points_per_wing(), dtype=np.int32)
        self.npts = int(self._ppw.sum())
        self.nseg = int((self._ppw - 1).sum())
        self.h = self.L.ora_create(C.byref(cfg), _dp(self._xy) if self._xy.size else None,
                                   self._ppw.ctypes.data_as(I) if self._ppw.size else None,
                                   nthreads)
        if not self.h:
            raise ValueError("oracle rejected the configuration")
        self.row_len = 4 + 12 * self.W
        if ep.motion is not None and motion_source == 1:
            self.set_motion_table(ep.motion)

    def close(self):
        if self.h:
            self.L.ora_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_motion_table(self, rows):
        rows = np.ascontiguousarray(rows, dtype=np.float64)
        rc = self.L.ora_set_motion_table(self.h, _dp(rows), rows.shape[0], rows.shape[1])
        if rc != 0:
            raise ValueError(f"motion table rejected ({rc})")

    def set_stream_rows(self, start, target):
        a = np.ascontiguousarray(start, dtype=np.float64)
        b = np.ascontiguousarray(target, dtype=np.float64)
        self.L.ora_set_stream_rows(self.h, _dp(a), _dp(b))

    def step(self, n: int) -> np.ndarray:
        row = np.zeros(self.row_len)
        rc = self.L.ora_step(self.h, n, _dp(row))
        if rc != 0:
            raise RuntimeError(f"oracle step {n} failed ({rc})")
        return row

    def run(self, first: int, count: int) -> np.ndarray:
        return np.stack([self.step(n) for n in range(first, first + count)]) if count else \
            np.zeros((0, self.row_len))

    def field(self, which) -> np.ndarray:
        names = {"rho": 0, "u": 1, "v": 2, "pre": 3, "u0": 4, "v0": 5, "gfx": 6, "gfy": 7}
        code = names[which] if isinstance(which, str) else int(which)
        out = np.zeros(self.nx * self.ny)
        if self.L.ora_get_field(self.h, code, _dp(out)) != 0:
            raise ValueError(which)
        return out.reshape(self.ny, self.nx)

    def f(self) -> np.ndarray:
        return np.stack([self.field(100 + k) for k in range(9)])

    def f0(self) -> np.ndarray:
        return np.stack([self.field(200 + k) for k in range(9)])

    def set_f(self, f):
        a = np.ascontiguousarray(f, dtype=np.float64)
        self.L.ora_set_f(self.h, _dp(a))

    def band(self) -> np.ndarray:
        n = C.c_int32(0)
        self.L.ora_get_band(self.h, C.byref(n), None, 0)
        out = np.zeros(3 * max(n.value, 1), dtype=np.int32)
        self.L.ora_get_band(self.h, C.byref(n), out.ctypes.data_as(I), n.value)
        return out[:3 * n.value].reshape(-1, 3)

    def markers(self):
        xb1, yb1 = np.zeros(self.npts), np.zeros(self.npts)
        xb2, yb2 = np.zeros(self.nseg), np.zeros(self.nseg)
        self.L.ora_get_markers(self.h, _dp(xb1), _dp(yb1), _dp(xb2), _dp(yb2))
        return xb1, yb1, xb2, yb2

    def sums(self):
        s = np.zeros(self.row_len)
        cnt, ln = C.c_int32(0), C.c_int32(0)
        self.L.ora_get_sums(self.h, _dp(s), C.byref(cnt), C.byref(ln))
        return s, cnt.value, ln.value

    def reset_sums(self):
        self.L.ora_reset_sums(self.h)

    def err(self) -> float:
        return self.L.ora_err(self.h)

    def tau(self) -> float:
        return self.L.ora_tau(self.h)

    def ibm_residual(self) -> float:
        return self.L.ora_ibm_residual(self.h)

    def move_mesh(self, dr: int):
        if self.L.ora_move_mesh(self.h, dr) != 0:
            raise ValueError(dr)

    def stream_row(self, t):
        row = np.zeros(1 + 9 * self.W)
        self.L.ora_stream_row(self.h, t, _dp(row))
        return row

    def build_stream_target_row(self, start, target_time, delta):
        a = np.ascontiguousarray(start, dtype=np.float64)
        d = np.ascontiguousarray(delta, dtype=np.float64)
        out = np.zeros(1 + 9 * self.W)
        rc = self.L.ora_build_stream_target_row(self.h, _dp(a), target_time, _dp(d), _dp(out))
        if rc != 0:
            raise ValueError("STEP time must not precede the segment start")
        return out


def delta_phi(r: float) -> float:
    return lib().ora_delta_phi(r)


def inverse_m() -> np.ndarray:
    out = np.zeros(81)
    lib().ora_inverse_m(_dp(out))
    return out.reshape(9, 9)


def interpolate_triplet(s0, v0, v1, dt, local_t):
    s, v, a = C.c_double(), C.c_double(), C.c_double()
    lib().ora_interpolate_triplet(s0, v0, v1, dt, local_t, C.byref(s), C.byref(v), C.byref(a))
    return s.value, v.value, a.value
