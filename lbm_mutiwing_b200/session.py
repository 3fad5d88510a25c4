"""One online episode: the per-episode part of the reference's ZeroMQ driver
(run_zmq_driver, reset_zmq_episode, advance_zmq_segment,
finalize_force_reply_average, save_current_flow_output; driver.f90:59-408)
over a ``Simulation`` (or any object with the same methods).

``EpisodeSession.handle`` takes one parsed command and returns the reply
text.  A session holds no socket: the single-client driver and the
multi-client server both feed it.
"""
from __future__ import annotations

import math
import os
from typing import Callable, Optional

import numpy as np

from . import protocol as P
from .api import STEP_FIELDS, finalize_force_average


def fortran_nint(x: float) -> int:
    """NINT: nearest integer, halves away from zero."""
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))


class EpisodeSession:
    """State of one client's episode between requests."""

    def __init__(self, sim, ep, out_dir: Optional[str] = None, episode_index: int = 0,
                 write_force_files: bool = False, output_stride=(2, 2), stepper=None):
        self.sim = sim
        # stepper(sim, n_steps, first_cycle=, rows=, flags=) advances the
        # simulation: by default its own step; the server passes its
        # continuous batcher
        self.stepper = stepper
        self.ep = ep
        self.W = ep.wing_count
        self.ncol = 1 + 9 * self.W
        self.out_dir = out_dir
        self.episode_index = episode_index
        self.write_force_files = write_force_files and out_dir is not None
        self.output_stride = output_stride
        self.active = False
        self.n = 1
        self.flag2 = 1
        self.start_row = np.zeros(self.ncol)
        self.target_row = np.zeros(self.ncol)
        self.motion_end_time = 0.0
        self.force_writer = None
        self.steps_run = 0            # lattice steps since the session began

    # -- commands
    def handle(self, cmd: P.Command) -> str:
        if cmd.kind == P.CMD_RESET:
            return self.reset(cmd.values[0])
        if cmd.kind == P.CMD_STEP:
            if not self.active:
                return P.error_reply(P.ERR_NEED_RESET_STEP)
            return self.step(cmd.values[0], cmd.values)
        if cmd.kind == P.CMD_OUTPUT:
            if not self.active:
                return P.error_reply(P.ERR_NEED_RESET_SAVE)
            return self.save()
        if cmd.kind == P.CMD_STOP:
            self.close()
            return P.status_reply(P.STATUS_STOPPING)
        return P.error_reply(P.ERR_EXPECTED)

    def reset(self, t: float) -> str:
        """RESET (driver.f90:113-141): a new episode at time 0 and its first step."""
        if abs(t) > 1.0e-12:
            return P.error_reply(P.ERR_RESET_NONZERO)
        self.episode_index += 1
        self.start_row = np.zeros(self.ncol)
        self.target_row = np.zeros(self.ncol)
        self.start_row[0] = t
        self.target_row[0] = t
        self.motion_end_time = t
        self._open_force_files()
        self.sim.reset()                      # reset_zmq_episode (driver.f90:205-258)
        self.n = 1
        self.flag2 = 1
        self.active = True
        err = self._advance(t)
        if err:
            self._close_force_files()
            self.active = False
            return P.error_reply(err)
        return self._force_reply()

    def step(self, t: float, values) -> str:
        """STEP (driver.f90:174-195)."""
        start = self.target_row.copy()
        try:
            nxt = self.sim.build_stream_target_row(start, t, np.asarray(values, dtype=np.float64))
        except Exception:
            return P.error_reply(P.ERR_STEP_BEFORE_START)
        prev_start, prev_target, prev_end = self.start_row, self.target_row, self.motion_end_time
        self.start_row, self.target_row, self.motion_end_time = start, nxt, t
        err = self._advance(t)
        if err:
            # driver.f90:188-191: the segment is not taken
            self.start_row, self.target_row, self.motion_end_time = prev_start, prev_target, prev_end
            return P.error_reply(err)
        return self._force_reply()

    def save(self) -> str:
        """SAVE (save_current_flow_output, driver.f90:291-320)."""
        if self.flag2 != 0:
            return P.error_reply(P.ERR_SAVE_TRANSITION)
        cycle = max(1, self.n - 1)
        if self.out_dir is not None:
            from .output import write_flow_field
            sx, sy = self.output_stride
            u, v, pre, vort = self.sim.output(sx, sy)
            xb1, yb1, _, _ = self.sim.markers()
            path = os.path.join(self.out_dir, f"episode_{self.episode_index}", f"F{cycle}.dat")
            write_flow_field(path, cycle, self.ep, u, v, pre, vort, sx, sy, xb1, yb1,
                             list(self.ep.points_per_wing()), 0)
        return P.status_reply(f"FLOW_SAVED F{cycle}.dat")

    def close(self):
        self._close_force_files()
        self.active = False

    # -- segment
    def _advance(self, target_time: float) -> Optional[str]:
        """advance_zmq_segment (driver.f90:322-363): steps n .. target cycle."""
        dt = self.ep.scale * self.ep.uu
        if dt <= 0.0:
            return P.ERR_DT
        target_cycle = fortran_nint(target_time / dt) + 1
        aligned = float(target_cycle - 1) * dt
        if abs(aligned - target_time) > 1.0e-10:
            return P.ERR_ALIGN
        if target_cycle < self.n:
            return P.ERR_BACKWARDS
        nsteps = target_cycle - self.n + 1
        self.sim.set_stream_rows(self.start_row, self.target_row)
        self.sim.reset_sums()
        if self.stepper is not None:
            rows = self.stepper(self.sim, nsteps, first_cycle=self.n, rows=True, flags=STEP_FIELDS)
        else:
            rows = self.sim.step(nsteps, first_cycle=self.n, rows=True, flags=STEP_FIELDS)
        self.last_rows = rows
        self.n = target_cycle + 1
        self.steps_run += nsteps
        # run_zmq_time_step: flag2 counts down after a lattice shift
        for _ in range(nsteps):
            if self.flag2 > 0:
                self.flag2 -= 1
        if self.force_writer is not None:
            self.force_writer.add(rows)
        return None

    def _force_reply(self) -> str:
        s, cnt, ln = self.sim.sums()
        row = finalize_force_average(s, cnt, ln, self.W, self.motion_end_time, self.last_rows[-1])
        return P.force_reply(row)

    def _open_force_files(self):
        self._close_force_files()
        if self.write_force_files:
            from .output import ForceWriter
            self.force_writer = ForceWriter(self.out_dir, self.episode_index, self.W,
                                            self.ep.wing_x_origin, self.ep.wing_x_spacing)

    def _close_force_files(self):
        if self.force_writer is not None:
            self.force_writer.close()
            self.force_writer = None
