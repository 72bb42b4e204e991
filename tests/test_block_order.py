"""Structured-block numbering of reorder 4 (host only): the half-cylinder O-grid, the ramp and the
box are recognised with the right extents and a numbering whose (i +- 1, j) and (i, j +- 1) cells
are the mesh's face neighbours; mixed meshes are refused."""
import numpy as np
import pytest

import cfd_solver_withcuda_b200 as cb


def check_block(m, ni, nj):
    got_ni, got_nj, lh, cells = m.block_order()
    assert (got_ni, got_nj) == (ni, nj)
    NP = m.n_physical
    assert sorted(cells.tolist()) == list(range(NP))
    grid = cells.reshape(nj, ni)
    nb = m.neighbours
    for j in range(nj):
        for i in range(ni):
            c = grid[j, i]
            want = set()
            for di, dj in ((1, 0), (-1, 0), (0, 1), (0, -1)):
                if 0 <= i + di < ni and 0 <= j + dj < nj:
                    want.add(int(grid[j + dj, i + di]))
            phys = {int(n) for n in nb[c, :m.n_faces[c]] if n < NP}
            assert phys == want, (i, j)
    return lh


def test_half_cylinder_block():
    # 1024 x 512 half cylinder: i runs around the body (the multiple of 32), natural numbering
    m = cb.Mesh.half_cylinder(64, 20, 1.0, 4.0, 1.005)
    check_block(m, 64, 20)
    assert np.array_equal(m.block_order()[3], np.arange(m.n_physical))


@pytest.mark.parametrize("nx,ny", [(52, 18), (64, 32), (33, 7)])
def test_ramp_block(nx, ny):
    m = cb.Mesh.ramp(nx, ny)
    # i is the side that is a multiple of 32 when only one is, else the longer side
    if (nx % 32 == 0) != (ny % 32 == 0):
        x_is_i = nx % 32 == 0
    else:
        x_is_i = nx >= ny
    check_block(m, *((nx, ny) if x_is_i else (ny, nx)))


def test_box_block():
    m = cb.Mesh.box(100, 4)
    check_block(m, 100, 4)


def test_mixed_mesh_is_refused():
    m = cb.Mesh.bump(40, 16, 3.0, 1.0, 0.1, 3, 0.3, 11, True)
    with pytest.raises(cb.CfdError):
        m.block_order()


def test_thin_block_is_refused():
    m = cb.Mesh.box(10, 1)
    with pytest.raises(cb.CfdError):
        m.block_order()
