"""The online text protocol of the reference's ZeroMQ driver.

Requests (zmq_comm.f90:224-279, parse_command_message):
  ``RESET [t]`` / ``START [t]``  new episode at time t (must be 0.0)
  ``STEP t d_1 .. d_3W``        advance to time t; per wing the increments of
                                 omega, x velocity and y velocity
  ``SAVE`` / ``OUTPUT``          write the flow field of the current step
  ``STOP`` / ``EXIT``            end
Replies: ``FORCE <n> v_1 .. v_n`` (es24.16 values, zmq_comm.f90:183-203),
``STATUS <text>``, ``ERROR <text>``.  The error and status texts are the
reference's own, byte for byte, so existing clients can match on them.

Extension: a token after RESET's time names the episode's workload (a
multi-client server serves episodes of different sizes); the reference's
list-directed read ignores such trailing tokens.
"""
from __future__ import annotations

import math
import re
from dataclasses import dataclass, field
from typing import List, Optional

CMD_RESET, CMD_STEP, CMD_OUTPUT, CMD_STOP = "RESET", "STEP", "OUTPUT", "STOP"

# reply texts of the reference (zmq_comm.f90, driver.f90, mode.f90)
ERR_PARSE = "无法解析 ZeroMQ 指令"
ERR_RESET_TIME = "RESET 指令缺少初始时间"
ERR_STEP_VALUES = "STEP 指令缺少目标时刻或速度增量"
ERR_UNKNOWN = "未知 ZeroMQ 指令: "
ERR_RESET_NONZERO = "RESET command must provide initial time 0.0"
ERR_NEED_RESET_STEP = "online mode requires RESET before STEP"
ERR_NEED_RESET_SAVE = "online mode requires RESET before SAVE"
ERR_EXPECTED = "expected STEP, SAVE, RESET or STOP"
ERR_STEP_BEFORE_START = "STEP 时间必须大于等于当前段起始时刻"
ERR_ALIGN = "STEP 时间必须与 LBM 时间步严格对齐"
ERR_BACKWARDS = "STEP 时间必须大于等于当前待推进时刻"
ERR_DT = "求解器时间步无效"
ERR_SAVE_TRANSITION = "当前时刻处于移网格后的过渡阶段，请在下一次 STEP 后再保存流场"
STATUS_STOPPING = "STOPPING"


class ProtocolError(ValueError):
    pass


@dataclass
class Command:
    kind: str
    values: List[float] = field(default_factory=list)
    workload: Optional[str] = None


_REAL = re.compile(r"^[+-]?(\d+\.?\d*|\.\d+)([eEdDqQ][+-]?\d+)?$")


def _real(tok: str) -> float:
    """A Fortran list-directed real (d and q exponents accepted)."""
    if not _REAL.match(tok):
        raise ValueError(tok)
    return float(re.sub(r"[dDqQ]", "e", tok))


def _tokens(text: str) -> List[str]:
    # list-directed input separates values by blanks or commas
    return [t for t in re.split(r"[\s,]+", text.strip()) if t]


def parse(text: str, wing_count: int) -> Command:
    """parse_command_message (zmq_comm.f90:224-279)."""
    toks = _tokens(text)
    if not toks:
        raise ProtocolError(ERR_PARSE)
    key = toks[0].upper()
    if key in ("RESET", "START"):
        if len(toks) == 1:
            return Command(CMD_RESET, [0.0])
        try:
            t = _real(toks[1])
        except ValueError:
            raise ProtocolError(ERR_RESET_TIME)
        return Command(CMD_RESET, [t], toks[2] if len(toks) > 2 else None)
    if key == "STEP":
        need = 1 + 3 * wing_count
        try:
            vals = [_real(x) for x in toks[1:1 + need]]
        except ValueError:
            raise ProtocolError(ERR_STEP_VALUES)
        if len(vals) < need:
            raise ProtocolError(ERR_STEP_VALUES)
        return Command(CMD_STEP, vals)
    if key in ("OUTPUT", "SAVE"):
        return Command(CMD_OUTPUT)
    if key in ("STOP", "EXIT"):
        return Command(CMD_STOP)
    raise ProtocolError(ERR_UNKNOWN + toks[0].upper())


def es24_16(x: float) -> str:
    """Fortran ES24.16, left-adjusted (trim(adjustl(token)))."""
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "-Infinity" if x < 0 else "Infinity"
    m, e = f"{x:.16E}".split("E")
    ev = int(e)
    return m + (f"E{'-' if ev < 0 else '+'}{abs(ev):02d}" if abs(ev) <= 99 else f"{'-' if ev < 0 else '+'}{abs(ev):03d}")


def force_reply(row) -> str:
    """zmq_send_force_reply: FORCE, the length, the values."""
    return "FORCE " + str(len(row)) + "".join(" " + es24_16(float(v)) for v in row)


def error_reply(text: str) -> str:
    return "ERROR " + text


def status_reply(text: str) -> str:
    return "STATUS " + text


def parse_force_reply(text: str) -> List[float]:
    toks = text.split()
    if not toks or toks[0] != "FORCE":
        raise ProtocolError(text)
    n = int(toks[1])
    vals = [float(x) for x in toks[2:2 + n]]
    if len(vals) != n:
        raise ProtocolError(text)
    return vals
