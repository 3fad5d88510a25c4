"""The C-ABI library loads on a CPU-only host and exports every entry point
that include/lbm_mutiwing.h declares (no compute calls)."""
import os
import re

from lbm_mutiwing_b200 import api, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "lbm_mutiwing.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(lbm_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_header_symbols():
    build.build()
    lib = api.load_library()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers the same set
    assert sorted(n for n, _, _ in api.SIGNATURES) == names


def test_abi_version_and_defaults():
    lib = api.load_library()
    assert lib.lbm_abi_version() == 1
    cfg = api.LbmConfig()
    lib.lbm_config_default(cfg)
    assert (cfg.nx, cfg.ny, cfg.wing_count) == (4001, 2001, 2)
    assert abs(cfg.ox + 20.0) < 1e-15 and abs(cfg.wing_y_origin - 0.5) < 1e-15


def test_create_fails_loudly_without_gpu_or_bad_config():
    """A bad configuration is refused with an error string (no exit)."""
    from lbm_mutiwing_b200 import workloads as wl
    ep = wl.Episode(name="bad", nx=3, ny=3, scale=0.01, re=100.0, ox=0.0, oy=0.0)
    try:
        api.Simulation(ep)
    except api.LbmError as e:
        assert "6 x 6" in str(e) or "CUDA" in str(e)
    else:
        raise AssertionError("expected LbmError")


def test_flag_constants_match_header_and_fortran_block():
    """Every LBM_FLAG_* / LBM_STEP_* / LBM_PRECISION_* macro of the header has
    the same value in the Python binding, and every flag the same value in
    the Fortran interface block of the integration notes."""
    hdr = open(os.path.join(ROOT, "include", "lbm_mutiwing.h")).read()
    macros = dict((m, int(v)) for m, v in re.findall(r"#define (LBM_(?:FLAG|STEP|PRECISION)_[A-Z0-9_]+)\s+(\d+)", hdr))
    assert {"LBM_FLAG_PASS_TALL_TILES", "LBM_FLAG_PASS_SHORT_TILES", "LBM_FLAG_SINGLE_STEPS"} <= set(macros)
    for m, v in macros.items():
        name = m[len("LBM_"):]
        if hasattr(api, name):
            assert getattr(api, name) == v, m
    flags = {m: v for m, v in macros.items() if m.startswith("LBM_FLAG_")}
    for m, v in flags.items():
        assert hasattr(api, m[len("LBM_"):]), m
    fortran = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    fvals = dict((m, int(v)) for m, v in re.findall(r"(LBM_FLAG_[A-Z0-9_]+) = (\d+)", fortran))
    assert fvals == flags
