"""Makes tests/golden/oracle_regression.json: a short oracle run on the
reference's own marker file (tests/golden/boundary.dat, a copy of the
reference's boundary.dat data) on a 2 x 1 chord lattice at dx = 0.01.

Run: python -m tests.golden.make_golden
"""
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def episode():
    from lbm_mutiwing_b200 import workloads as wl
    pts = wl.read_boundary_file(os.path.join(HERE, "boundary.dat"))
    nx, ny, ox, oy = wl.lattice(2.0, 1.0, 0.01)
    ep = wl.Episode(name="golden", nx=nx, ny=ny, scale=0.01, re=500.0, ox=ox, oy=oy,
                    wing_x_origin=-0.4, wing_x_spacing=1.5, wing_y_origin=0.0, steps=12)
    ep.markers = [pts]
    mo = wl.WingMotion(x=-0.4, y=0.0, pitch_amp=0.2, heave_amp=0.05, freq=2.0)
    ep.motion = wl.motion_table([mo], 13 * ep.scale * ep.uu, ep.scale * ep.uu)
    return ep


def run_case(oracle_mod):
    ep = episode()
    o = oracle_mod.Oracle(ep)
    rows = o.run(1, ep.steps)
    f = o.f()
    return {"rows": rows.tolist(), "band_n": int(o.band().shape[0]),
            "f_sum": float(np.sum(f)), "u_sum": float(np.sum(o.field("u"))),
            "v_sum": float(np.sum(o.field("v")))}


if __name__ == "__main__":
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from oracle import oracle
    oracle.build()
    out = run_case(oracle)
    with open(os.path.join(HERE, "oracle_regression.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print("band", out["band_n"], "rows", len(out["rows"]))
