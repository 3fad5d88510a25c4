"""Synthetic inputs for the benchmark configurations: NACA 4-digit marker
loops, analytic pitch/heave motion tables and lattice configurations.

Marker files in the reference (``boundary.dat``, read at airfoil.f90:229 with
format ``2f14.8``) hold a closed loop of points in the body frame, starting at
the leading edge, running over the upper surface to the trailing edge and back
along the lower surface, with the first point repeated at the end; chord 1
with the pitch axis at the quarter chord (x in [-0.25, 0.75]).  ``naca_loop``
writes the same layout.  A wing with ``n`` markers here has ``n`` segments
(``n + 1`` points): the immersed-boundary forcing acts at segment midpoints
(airfoil.f90:267-270), so segments are the Lagrangian markers.

Motion tables follow ``motion_params.dat`` (mode.f90:104-178): column 1 is
time, then per wing ``angle omega omgac x xv xa y yv ya`` with absolute x, y.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Sequence

import numpy as np

PAI = 3.1415926535897932384626433832795  # main.f90:9


def naca_loop(thickness: float, n_markers: int, spacing: str = "arc") -> np.ndarray:
    """Closed NACA 00xx loop, shape (n_markers + 1, 2), body frame.

    The symmetric 4-digit thickness law with the closed-trailing-edge
    coefficient (-0.1036) gives one shared trailing-edge point.  ``spacing`` is
    ``"arc"`` (equal arc length along each surface; the default),
    ``"uniform"`` (uniform x, the style of the reference's shipped
    boundary.dat) or ``"cosine"`` (x = (1 - cos b) / 2, b uniform).  At 200
    markers on a chord of 100 nodes, arc spacing puts markers 1.0-1.02
    lattice spacings apart everywhere; cosine spacing puts trailing-edge
    markers 0.025 spacings apart, where the immersed-boundary system becomes
    numerically singular and the reference's algorithm (the FP64 oracle)
    diverges after about 1150 steps of the 800x400 case; uniform-x spacing
    leaves leading-edge gaps of 2 spacings.  Arc and uniform-x spacing both
    run 2000 steps of that case stably.
    """
    if n_markers < 4:
        raise ValueError("need at least 4 markers per wing")
    nh = n_markers // 2
    nl = n_markers - nh

    def xs(k, m):
        b = np.arange(k + 1) / m
        if spacing == "cosine":
            return 0.5 * (1.0 - np.cos(np.pi * b))
        if spacing == "uniform":
            return b
        raise ValueError("spacing must be 'cosine', 'uniform' or 'arc'")

    def yt(x):
        return 5.0 * thickness * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2
                                  + 0.2843 * x ** 3 - 0.1036 * x ** 4)

    if spacing == "arc":
        # equal arc length along each surface: a fine cosine sampling of the
        # surface resampled at equal steps (both ends kept exactly)
        xf = 0.5 * (1.0 - np.cos(np.pi * np.linspace(0.0, 1.0, 64 * n_markers + 1)))
        yf = yt(xf)
        s = np.concatenate([[0.0], np.cumsum(np.hypot(np.diff(xf), np.diff(yf)))])

        def surface(m):
            t = np.linspace(0.0, s[-1], m + 1)
            return np.interp(t, s, xf), np.interp(t, s, yf)
        xu, yu = surface(nh)
        xl, yl = surface(nl)
        x = np.concatenate([xu, xl[::-1][1:]])
        y = np.concatenate([yu, -yl[::-1][1:]])
    else:
        xu = xs(nh, nh)                     # LE .. TE, nh + 1 points
        xl = xs(nl, nl)[::-1][1:]           # TE(excluded) .. LE, nl points
        x = np.concatenate([xu, xl])
        y = np.concatenate([yt(xu), -yt(xl)])
    y[-1] = 0.0
    pts = np.stack([x - 0.25, y], axis=1)
    pts[-1] = pts[0]
    return pts


@dataclasses.dataclass
class WingMotion:
    """Analytic pitch/heave motion of one wing (angles in radians)."""
    x: float                 # absolute x of the pitch axis
    y: float                 # mean absolute y of the pitch axis
    pitch_amp: float = 15.0 * math.pi / 180.0
    heave_amp: float = 0.5
    freq: float = 0.5
    phase: float = 0.0       # added to both pitch and heave phase

    def row(self, t: np.ndarray) -> np.ndarray:
        om = 2.0 * math.pi * self.freq
        ph = om * t + self.phase
        th = self.pitch_amp * np.sin(ph)
        thd = self.pitch_amp * om * np.cos(ph)
        thdd = -self.pitch_amp * om * om * np.sin(ph)
        hp = ph + 0.5 * math.pi
        y = self.y + self.heave_amp * np.sin(hp)
        yv = self.heave_amp * om * np.cos(hp)
        ya = -self.heave_amp * om * om * np.sin(hp)
        z = np.zeros_like(t)
        return np.stack([th, thd, thdd, z + self.x, z, z, y, yv, ya], axis=1)


def motion_table(wings: Sequence[WingMotion], t_end: float, dt: float = 1.0e-4) -> np.ndarray:
    """Rows (t, 9 columns per wing) sampled every ``dt`` on [0, t_end]."""
    n = int(round(t_end / dt)) + 1
    t = np.arange(n) * dt
    cols = [t[:, None]] + [w.row(t) for w in wings]
    return np.concatenate(cols, axis=1)


@dataclasses.dataclass
class Episode:
    """Everything needed to create one simulation: lattice, geometry, motion."""
    name: str
    nx: int
    ny: int
    scale: float
    re: float
    ox: float
    oy: float
    uu: float = 0.01
    wing_x_origin: float = 0.0
    wing_x_spacing: float = 1.5
    wing_y_origin: float = 0.5
    markers: List[np.ndarray] = dataclasses.field(default_factory=list)
    motion: np.ndarray | None = None
    steps: int = 0
    # draws of a seeded workload that the domain's size capped (mixed_batch)
    meta: dict = dataclasses.field(default_factory=dict)

    @property
    def wing_count(self) -> int:
        return len(self.markers)

    @property
    def nodes(self) -> int:
        return self.nx * self.ny

    def markers_xy(self) -> np.ndarray:
        if not self.markers:
            return np.zeros((0, 2))
        return np.ascontiguousarray(np.concatenate(self.markers, axis=0), dtype=np.float64)

    def points_per_wing(self) -> np.ndarray:
        return np.array([m.shape[0] for m in self.markers], dtype=np.int32)


def lattice(width: float, height: float, scale: float):
    """Node counts and centred origin exactly as ini_mesh.f90:22-23, 36-37."""
    nx = int(round(width / scale)) + 1
    ny = int(round(height / scale)) + 1
    return nx, ny, -0.5 * width, -0.5 * height


def tandem_pitch_heave(name: str, width: float, height: float, scale: float, re: float,
                       x_first: float, y: float, n_markers: int, steps: int,
                       thickness: float = 0.12, lag: float = 0.25 * math.pi,
                       spacing: str = "arc", n_wings: int = 2, x_spacing: float = 1.5,
                       pitch_deg: float = 15.0, heave: float = 0.5, freq: float = 0.5) -> Episode:
    """Tandem wings with the analytic pitch/heave law of the benchmark configs.

    ``x_first``/``y`` are in the reference's centred frame.  Wing k lags wing
    k-1 by ``lag`` in phase.
    """
    nx, ny, ox, oy = lattice(width, height, scale)
    ep = Episode(name=name, nx=nx, ny=ny, scale=scale, re=re, ox=ox, oy=oy,
                 wing_x_origin=x_first, wing_x_spacing=x_spacing, wing_y_origin=y,
                 steps=steps)
    ep.markers = [naca_loop(thickness, n_markers, spacing) for _ in range(n_wings)]
    wings = [WingMotion(x=x_first + k * x_spacing, y=y, pitch_amp=pitch_deg * math.pi / 180.0,
                        heave_amp=heave, freq=freq, phase=-k * lag) for k in range(n_wings)]
    dt = scale * ep.uu
    ep.motion = motion_table(wings, (steps + 1) * dt, dt)
    return ep


def tandem_800x400(steps: int = 2000, scale_factor: int = 1) -> Episode:
    """800x400 lattice (8x4 chords, dx = 0.01), Re 200, NACA0012 tandem at
    corner-frame x = 2.0 / 3.5, y = 2.0 (centred frame -2.0 / -0.5, 0.0),
    200 markers per wing at equal arc length (see naca_loop).  ``scale_factor`` > 1 coarsens the
    lattice for quick tests (dx = 0.01 * scale_factor)."""
    return tandem_pitch_heave("tandem_800x400_re200", 8.0, 4.0, 0.01 * scale_factor, 200.0,
                              -2.0, 0.0, 200 // scale_factor, steps)


def tandem_4000x2000(steps: int = 10000) -> Episode:
    """4000x2000 lattice (40x20 chords, dx = 0.01), Re 1000, NACA0012 at the
    reference's default wing offsets x = 0.0 / 1.5, y = 0.5, 200 markers."""
    return tandem_pitch_heave("tandem_4000x2000_re1000", 40.0, 20.0, 0.01, 1000.0,
                              0.0, 0.5, 200, steps)


def formation_16000x8000(steps: int = 20000) -> Episode:
    """16000x8000 lattice (dx = 0.0025), Re 5000, four NACA0012 wings with 800
    markers each in a 2x2 staggered formation (absolute positions set through
    the motion table's x and y columns)."""
    nx, ny, ox, oy = lattice(40.0, 20.0, 0.0025)
    ep = Episode(name="formation_16000x8000_re5000", nx=nx, ny=ny, scale=0.0025, re=5000.0,
                 ox=ox, oy=oy, wing_x_origin=0.0, wing_x_spacing=1.5, wing_y_origin=0.5,
                 steps=steps)
    ep.markers = [naca_loop(0.12, 800) for _ in range(4)]
    pos = [(0.0, 1.0), (0.75, -0.25), (1.5, 1.0), (2.25, -0.25)]
    wings = [WingMotion(x=x, y=y, phase=-k * 0.25 * math.pi) for k, (x, y) in enumerate(pos)]
    dt = ep.scale * ep.uu
    ep.motion = motion_table(wings, (steps + 1) * dt, dt)
    return ep


def mixed_batch(count: int = 64, seed: int = 20261203, steps: int = 1000) -> List[Episode]:
    """Mixed batch: grids from {400x200, 800x400, 1200x600, 2000x1000}
    nodes at dx = 0.01, 1-4 NACA00xx wings (thickness 8-18 %, 100-300
    markers), pitch 5-25 deg, heave 0.1-0.6 chord, f 0.2-1.0, seeded.

    Wings sit 1.5 chords apart, leading edge at least 0.75 chord from the
    inflow border and trailing edge 1.25 chords from the outflow border, so
    the draw of 1-4 wings is capped by what the domain holds (two wings in
    a 4-chord domain); the heave amplitude is capped at 0.3 h - 0.5 so the
    wings stay clear of the top and bottom borders in the 2-chord-high grids."""
    rng = np.random.default_rng(seed)
    sizes = [(4.0, 2.0), (8.0, 4.0), (12.0, 6.0), (20.0, 10.0)]
    eps = []
    for e in range(count):
        w, h = sizes[int(rng.integers(0, 4))]
        nw_draw = int(rng.integers(1, 5))
        spacing_x = 1.5
        lo, hi = -0.5 * w + 1.0, 0.5 * w - 2.0        # quarter-chord positions that fit
        nw = max(1, min(nw_draw, int((hi - lo) / spacing_x) + 1))
        x0 = lo
        nx, ny, ox, oy = lattice(w, h, 0.01)
        ep = Episode(name=f"mix{e:02d}", nx=nx, ny=ny, scale=0.01, re=float(rng.uniform(200, 1000)),
                     ox=ox, oy=oy, wing_x_origin=x0, wing_x_spacing=spacing_x, wing_y_origin=0.0,
                     steps=steps)
        th = float(rng.uniform(0.08, 0.18))
        nm = int(rng.integers(100, 301))
        ep.markers = [naca_loop(th, nm) for _ in range(nw)]
        wings = []
        heave_capped = 0
        for k in range(nw):
            pitch = float(rng.uniform(5, 25)) * math.pi / 180.0
            heave_draw = float(rng.uniform(0.1, 0.6))
            heave_capped += heave_draw > 0.3 * h - 0.5
            wings.append(WingMotion(x=x0 + k * spacing_x, y=0.0, pitch_amp=pitch,
                                    heave_amp=min(heave_draw, 0.3 * h - 0.5),
                                    freq=float(rng.uniform(0.2, 1.0)),
                                    phase=float(rng.uniform(0, 2 * math.pi))))
        ep.meta = {"wings_drawn": nw_draw, "wings_placed": nw, "heave_capped": int(heave_capped)}
        ep.motion = motion_table(wings, (steps + 1) * 0.01 * ep.uu, 0.01 * ep.uu)
        eps.append(ep)
    return eps


def read_boundary_file(path: str) -> np.ndarray:
    """Parse a reference marker file (two columns, ``2f14.8``)."""
    return np.loadtxt(path, dtype=np.float64).reshape(-1, 2)


def read_motion_file(path: str, wing_count: int) -> np.ndarray:
    """Parse a ``motion_params.dat`` table with ``1 + 9 * wing_count`` columns,
    skipping blank lines (mode.f90:124-158)."""
    rows = []
    with open(path) as fh:
        for line in fh:
            if not line.strip():
                continue
            vals = [float(v) for v in line.split()]
            if len(vals) < 1 + 9 * wing_count:
                raise ValueError(f"motion row needs {1 + 9 * wing_count} columns")
            rows.append(vals[:1 + 9 * wing_count])
    if not rows:
        raise ValueError("motion table is empty")
    return np.asarray(rows, dtype=np.float64)


_MIX_CACHE: dict = {}


def by_name(name: str, steps: int = 8) -> Episode:
    """Episode of a named workload for an online server: ``800x400``,
    ``4000x2000``, ``16000x8000``, or ``mix:<k>`` (episode k of the seeded
    64-episode mixed batch).  Online episodes take their motion from the
    clients, so the motion table is kept short."""
    if name == "800x400":
        return tandem_800x400(steps=steps)
    if name == "4000x2000":
        return tandem_4000x2000(steps=steps)
    if name == "16000x8000":
        return formation_16000x8000(steps=steps)
    if name.startswith("mix:"):
        k = int(name[4:])
        if "mix" not in _MIX_CACHE:
            _MIX_CACHE["mix"] = mixed_batch(64, steps=steps)
        return _MIX_CACHE["mix"][k]
    raise ValueError(f"unknown workload {name!r}")
