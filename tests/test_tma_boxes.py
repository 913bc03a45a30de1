"""The TMA box origins of the stage kernels, restated and checked on the CPU
(porturb_b200/csrc/dycore_kernels.cuh: k_xy step 0-1, k_zt step 1).

k_xy stages the cross of a 16x16 FP32 tile -- the tile, 5 rows above and
below, 5 columns left and right -- in five boxes of one 4-D map each: the
interior (16x16) at (i0, j0), the rows above (16x5) at j0-5 (ny-5 for the
first tile row), the rows below at j0+16 (0 for the last), the columns left
(8x16) at i0-8 (nx-8 for the first tile column) and right at i0+16 (0 for
the last).  A tile is staged only when it lies whole in the domain, the grid
is 3-D, and every box it needs exists (a precursor edge, or a halo box that
would straddle the domain's edge, keeps the threads' loads).  For every
staged tile of every grid here:

* every box's x origin is a multiple of 4 elements (16 bytes: the rule the
  hardware does not check before the copy runs);
* every box lies inside the tensor (no fill value is read as data);
* every cell of the cross comes from the box cell holding the global cell
  the threads' path reads (periodic wrap, precursor clamp).

k_zt's boxes start at (i0, j, k0-5) and (i0, j, k0) with i0 a multiple of 8;
a level's row in the halo box is its level minus k0-5, used only inside the
box (the threads load the rest), so every row it reads holds the level the
threads' path reads.
"""
import pytest

TX = TY = 16
PERIODIC, PRECURSOR = "periodic", "precursor"


def wrap(i, n):
    return i % n


def clamp(i, n):
    return min(max(i, 0), n - 1)


def xy_boxes(i0, j0, nx, ny, bc_x, bc_y):
    """The origins k_xy uses for the tile at (i0, j0), or None when the tile
    keeps the threads' loads."""
    if not (i0 + TX <= nx and j0 + TY <= ny and ny > 1):
        return None
    px, py = bc_x != PRECURSOR, bc_y != PRECURSOR
    xw = i0 - 8 if i0 > 0 else (nx - 8 if px else -1)
    xe = (i0 + TX if i0 + TX + 8 <= nx else -1) if i0 + TX < nx else (0 if px else -1)
    yn = j0 - 5 if j0 > 0 else (ny - 5 if py else -1)
    ys = (j0 + TY if j0 + TY + 5 <= ny else -1) if j0 + TY < ny else (0 if py else -1)
    if min(xw, xe, yn, ys) < 0:
        return None
    return {"in": (i0, j0, 16, 16), "top": (i0, yn, 16, 5), "bot": (i0, ys, 16, 5),
            "west": (xw, j0, 8, 16), "east": (xe, j0, 8, 16)}


def staged_source(r, c, i0, j0, boxes):
    """The global cell a staged cross cell (row r, column c of the 26x26
    cross, the tile at r, c = 5..20) is read from."""
    if r < 5:
        x, y = boxes["top"][0], boxes["top"][1]
        return x + (c - 5), y + r
    if r >= 5 + TY:
        x, y = boxes["bot"][0], boxes["bot"][1]
        return x + (c - 5), y + (r - 5 - TY)
    if c < 5:
        x, y = boxes["west"][0], boxes["west"][1]
        return x + (c + 3), y + (r - 5)
    if c >= 5 + TX:
        x, y = boxes["east"][0], boxes["east"][1]
        return x + (c - 5 - TX), y + (r - 5)
    x, y = boxes["in"][0], boxes["in"][1]
    return x + (c - 5), y + (r - 5)


def cross_cells():
    # Rows 5..20 with every column, rows 0..4 and 21..25 with columns 5..20.
    for r in range(5, 5 + TY):
        for c in range(TX + 10):
            yield r, c
    for r in list(range(5)) + list(range(5 + TY, TY + 10)):
        for c in range(5, 5 + TX):
            yield r, c


GRIDS = [(16, 16), (20, 24), (32, 32), (48, 37), (52, 40), (64, 48), (96, 64), (256, 80)]


@pytest.mark.parametrize("bc_y", [PERIODIC, PRECURSOR])
@pytest.mark.parametrize("bc_x", [PERIODIC, PRECURSOR])
@pytest.mark.parametrize("nx,ny", GRIDS)
def test_xy_boxes_aligned_inside_and_reading_the_threads_cells(nx, ny, bc_x, bc_y):
    assert nx % 4 == 0      # the maps exist only then (encode_state)
    xf = wrap if bc_x == PERIODIC else clamp
    yf = wrap if bc_y == PERIODIC else clamp
    staged = 0
    for j0 in range(0, ny, TY):
        for i0 in range(0, nx, TX):
            boxes = xy_boxes(i0, j0, nx, ny, bc_x, bc_y)
            if boxes is None:
                continue
            staged += 1
            for name, (x, y, bw, bh) in boxes.items():
                assert x % 4 == 0, (name, x)
                assert 0 <= x and x + bw <= nx and 0 <= y and y + bh <= ny, (name, x, y, nx, ny)
            for r, c in cross_cells():
                gi, gj = i0 - 5 + c, j0 - 5 + r
                assert staged_source(r, c, i0, j0, boxes) == (xf(gi, nx), yf(gj, ny)), (i0, j0, r, c)
    if bc_x == bc_y == PERIODIC and nx % TX == 0 and ny % TY == 0:
        assert staged == (nx // TX) * (ny // TY)     # every tile is staged
    # (nx = 52: the last whole tile's right box would straddle the edge, so
    # that tile keeps the threads' loads; so do partial tiles.)


def test_xy_tiles_at_precursor_edges_keep_thread_loads():
    nx, ny = 64, 64
    assert xy_boxes(0, 16, nx, ny, PRECURSOR, PERIODIC) is None
    assert xy_boxes(48, 16, nx, ny, PRECURSOR, PERIODIC) is None
    assert xy_boxes(16, 16, nx, ny, PRECURSOR, PERIODIC) is not None
    assert xy_boxes(16, 0, nx, ny, PERIODIC, PRECURSOR) is None


ZT_X, ZT_Z = 8, 32


@pytest.mark.parametrize("nz,wall", [(40, True), (40, False), (64, True), (96, False), (128, True), (20, True)])
@pytest.mark.parametrize("nx", [8, 20, 64])
def test_zt_boxes(nx, nz, wall):
    hz = ZT_Z + 10
    for k0 in range(0, nz, ZT_Z):
        for i0 in range(0, nx, ZT_X):
            assert i0 % 4 == 0
            for p in range(k0 - 5, k0 + ZT_Z + 5):
                lv = p if 0 <= p < nz else (clamp(p, nz) if wall else wrap(p, nz))
                rr = lv - (k0 - 5)
                if 0 <= rr < hz:
                    # The box row rr holds level k0 - 5 + rr = lv, inside the tensor.
                    assert k0 - 5 + rr == lv and 0 <= lv < nz
