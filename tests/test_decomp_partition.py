"""The interior/edge split of a decomposed tile's x/y kernel, restated and
checked on the CPU (Impl::dec_interior and the edge launches of
Impl::stage in porturb_b200/csrc/impl.cuh).

The interior tiles [tx0, tx1) x [ty0, ty1) run while the halos cross; the
edge tiles are four rectangles launched after the exchange: the rows below
and above the interior (every column), then the columns left and right of
it (the interior's rows).  For every tile size here: the interior and the
four rectangles cover every 16x16 tile of the decomposed tile exactly once,
and no interior tile's cross (the tile and 5 cells around it) reaches
beyond the decomposed tile, so none of them reads a halo slab.
"""
import pytest

T = 16


def blocks(n):
    return (n + T - 1) // T


def interior(nx, ny):
    tx0 = ty0 = 1
    tx1 = max(tx0, (nx - T - 5) // T + 1) if nx >= T + 5 else tx0
    ty1 = max(ty0, (ny - T - 5) // T + 1) if ny >= T + 5 else ty0
    return tx0, tx1, ty0, ty1


def edge_rects(nx, ny):
    tx0, tx1, ty0, ty1 = interior(nx, ny)
    nbx, nby = blocks(nx), blocks(ny)
    return [(0, nbx, 0, ty0), (0, nbx, ty1, nby), (0, tx0, ty0, ty1), (tx1, nbx, ty0, ty1)]


def tiles_of(rect):
    x0, x1, y0, y1 = rect
    return [(x, y) for y in range(y0, y1) for x in range(x0, x1)]


@pytest.mark.parametrize("nx", [16, 20, 36, 37, 48, 52, 64, 100, 128])
@pytest.mark.parametrize("ny", [16, 21, 37, 56, 64, 128])
def test_interior_and_edges_partition_the_tiles(nx, ny):
    tx0, tx1, ty0, ty1 = interior(nx, ny)
    inner = tiles_of((tx0, tx1, ty0, ty1)) if tx1 > tx0 and ty1 > ty0 else []
    edges = [t for r in edge_rects(nx, ny) for t in tiles_of(r)] if inner else \
        tiles_of((0, blocks(nx), 0, blocks(ny)))
    every = inner + edges
    assert len(every) == len(set(every)) == blocks(nx) * blocks(ny)
    for x, y in inner:
        i0, j0 = x * T, y * T
        assert i0 - 5 >= 0 and i0 + T + 5 <= nx and j0 - 5 >= 0 and j0 + T + 5 <= ny, (x, y)


def test_interior_sizes():
    assert interior(36, 64)[:2] == (1, 1)      # 1 + 16 + 5 > 36 - 16: no interior column
    assert interior(37, 64)[:2] == (1, 2)
    assert interior(64, 56) == (1, 3, 1, 3)
    assert interior(128, 128) == (1, 7, 1, 7)
