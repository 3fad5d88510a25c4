"""Makes tests/golden/motion_params_window.dat: a window of the reference's
own offline motion table (motion_params.dat, read by load_motion_table,
mode.f90:104-178) for a reduced-size regression run.

The reference table holds 220001 rows at 1e-4 time steps (t = 0 .. 22): both
wings stay at rest until t = 2, then pitch by +-45 degrees and heave by
+-0.5 chord with period 2.  The window is the rows from t = 2.25 (both wings
pitching and heaving) for 400 steps at dt = 1e-4 plus a margin, with the
time column re-based to start at 0; every other column is kept as the
reference wrote it (the same text format, one row per line).

Run (needs the reference's file): python -m tests.golden.make_motion_fixture
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SOURCE = "/root/reference/motion_params.dat"
FIRST_ROW = 22500        # t = 2.25
ROWS = 441               # t = 0 .. 0.044 after re-basing
OUT = os.path.join(HERE, "motion_params_window.dat")


def main():
    rows = []
    with open(SOURCE) as fh:
        for k, line in enumerate(fh):
            if k < FIRST_ROW:
                continue
            if len(rows) == ROWS:
                break
            if line.strip():
                rows.append([float(v) for v in line.split()])
    a = np.asarray(rows)
    a[:, 0] -= a[0, 0]
    with open(OUT, "w") as fh:
        for r in a:
            fh.write(" ".join(f"{v:.8f}" for v in r) + "\n")
    print(OUT, a.shape)


if __name__ == "__main__":
    sys.exit(main())
