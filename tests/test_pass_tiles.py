"""Index arithmetic of the two-step pass (CPU; the kernels' formulas restated).

The pass kernels rely on these invariants, which the GPU tests exercise only
on the lattices they run:
* the count kernel flags exactly the tiles whose R1 (the tile and one ring)
  holds a claimed node (``flag_pass_tiles`` in ibm.cu);
* every interior node is an output of exactly one tile;
* a tile off the border (``pass_border_tile``) has its R1 inside the
  interior and its pulls inside the lattice, and every tile's staged box
  starts on a 16-byte boundary;
* the ring kernel covers every interior node the far field reads;
* a support box touches at most ``pass_tiles_per_segment`` tiles (the near
  kernel's capacity per segment).
Both tile shapes a handle may take (``PASS_TY`` and ``PASS_TY_TALL`` rows)
are read from the header that sets them.
"""
import itertools
import os
import random
import re

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
HDR = os.path.join(HERE, "..", "lbm_mutiwing_b200", "csrc", "lbm_kernels.h")


def _shapes():
    s = open(HDR).read()
    tx = int(re.search(r"#define LBM_PASS_TX (\d+)", s).group(1))
    ty = int(re.search(r"#define LBM_PASS_TY (\d+)", s).group(1))
    tall = int(re.search(r"#define LBM_PASS_TY_TALL (\d+)", s).group(1))
    return [(tx, ty), (tx, tall)]


SHAPES = _shapes()
TX, TY = SHAPES[0]


def ntx(nx):
    return (nx + TX - 1) // TX


def nty(ny):
    return (ny - 2 + TY - 1) // TY


def border_tile(tx, ty, nx, ny):
    x0, y0 = tx * TX, 1 + ty * TY
    return x0 - 1 <= 0 or x0 + TX >= nx - 1 or y0 - 1 <= 0 or y0 + TY >= ny - 1


def flagged(i, j, nx, ny):
    tx0, tx1 = max(0, (i + TX - 1) // TX - 1), min(ntx(nx) - 1, (i + 1) // TX)
    ty0, ty1 = max(0, (j + TY - 2) // TY - 1), min(nty(ny) - 1, j // TY)
    return {(tx, ty) for tx in range(tx0, tx1 + 1) for ty in range(ty0, ty1 + 1)}


def in_r1(tx, ty, i, j):
    x0, y0 = tx * TX, 1 + ty * TY
    return x0 - 1 <= i <= x0 + TX and y0 - 1 <= j <= y0 + TY


LATTICES = [(27, 19), (201, 101), (385, 193), (130, 66)]


@pytest.fixture(params=SHAPES, ids=lambda s: "%dx%d" % s)
def shape(request):
    """The tile shape the formulas above use (module globals, as in the
    kernels' compile-time constants)."""
    g = globals()
    old = g["TX"], g["TY"]
    g["TX"], g["TY"] = request.param
    yield request.param
    g["TX"], g["TY"] = old


@pytest.mark.parametrize("nx,ny", LATTICES)
def test_flags_and_partition(shape, nx, ny):
    rng = random.Random(nx * 7 + ny)
    for _ in range(400):   # band nodes keep 3 nodes off the border
        i, j = rng.randrange(3, nx - 3), rng.randrange(3, ny - 3)
        want = {(tx, ty) for tx in range(ntx(nx)) for ty in range(nty(ny)) if in_r1(tx, ty, i, j)}
        assert flagged(i, j, nx, ny) == want, (i, j)
    owner = {}
    for tx in range(ntx(nx)):
        for ty in range(nty(ny)):
            x0, y0 = tx * TX, 1 + ty * TY
            assert (x0 - 4) % 4 == 0   # the box's first column on a 16-byte boundary
            for i, j in itertools.product(range(x0, x0 + TX), range(y0, y0 + TY)):
                if 1 <= i <= nx - 2 and 1 <= j <= ny - 2:
                    assert (i, j) not in owner
                    owner[(i, j)] = (tx, ty)
            if not border_tile(tx, ty, nx, ny):
                assert x0 - 1 >= 1 and x0 + TX <= nx - 2 and y0 - 1 >= 1 and y0 + TY <= ny - 2
                assert x0 - 2 >= 0 and x0 + TX + 1 <= nx - 1 and y0 - 2 >= 0 and y0 + TY + 1 <= ny - 1
    assert len(owner) == (nx - 2) * (ny - 2)


@pytest.mark.parametrize("nx,ny", LATTICES)
def test_ring_covers_far_field_reads(shape, nx, ny):
    ring = set()
    for u in range(6 * (ny - 2)):
        col = u // (ny - 2)
        ring.add((1 + col if col < 3 else nx - 7 + col, 1 + u % (ny - 2)))
    for u in range(4 * (nx - 8)):
        row = u // (nx - 8)
        ring.add((4 + u % (nx - 8), 1 + row if row < 2 else ny - 5 + row))
    need = set()
    for j in range(1, ny - 1):   # the columns next to the left and right borders
        for ic in (1, 2, nx - 2, nx - 3):
            need |= {(ic + a, j + b) for a, b in itertools.product((-1, 0, 1), repeat=2)}
    for i in range(nx):          # the rows next to the bottom and top borders
        for jc in (1, ny - 2):
            need |= {(i + a, jc + b) for a, b in itertools.product((-1, 0, 1), repeat=2)}
    need = {(i, j) for i, j in need if 1 <= i <= nx - 2 and 1 <= j <= ny - 2}
    assert need <= ring


def test_tiles_per_segment_bound(shape):
    per = ((8 + TX - 1) // TX + 1) * ((8 + TY - 1) // TY + 1)
    worst = 0
    for i1, j1 in itertools.product(range(3, 3 + 2 * TX), range(3, 3 + 2 * TY)):
        tiles = set()
        for i, j in itertools.product(range(i1, i1 + 6), range(j1, j1 + 6)):
            tiles |= flagged(i, j, 10 ** 6, 10 ** 6)
        worst = max(worst, len(tiles))
    assert worst <= per
