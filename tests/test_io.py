"""Solution files in the reference's formats: the VTK grid copy and the appended cell data are
byte-identical to the reference's Read_Write_Grid / Append_Solution on the same inputs (the
solution file itself written by the reference's Write_Solution)."""
import os

import numpy as np
import pytest

import cfd_solver_withcuda_b200 as cb
from cases import CASES, make_mesh, ref_params
from conftest import load_golden


def test_vtk_grid_and_solution_append_match_reference(tmp_path):
    from oracle import refpy
    if not refpy.ref_available():
        pytest.skip("oracle/_ref/libcfdref.so not built (reference sources absent at build time)")
    case = CASES["cyl_roe2_lts"]
    m = make_mesh(case)
    g = load_golden("cyl_roe2_lts")
    r = refpy.RefRun(m, ref_params(case))
    r.set_state(g["U0"])
    r.iterate(5)
    sol = str(tmp_path / "sol.txt")
    r.L.refh_write_solution(sol.encode())
    grid = str(tmp_path / "grid.vtk")
    m.write_vtk(grid)
    ref_out, mine = str(tmp_path / "ref.vtk"), str(tmp_path / "mine.vtk")
    r.L.refh_read_write_grid(grid.encode(), ref_out.encode())
    r.L.refh_append_solution(sol.encode(), ref_out.encode())
    cb.vtk_copy_grid(grid, mine)
    cb.vtk_append_solution(sol, mine)
    a, b = open(ref_out, "rb").read(), open(mine, "rb").read()
    assert len(a) > 1000 and a == b


def test_io_errors_are_status_codes(tmp_path):
    with pytest.raises(cb.CfdError) as e:
        cb.vtk_copy_grid(str(tmp_path / "missing.vtk"), str(tmp_path / "o.vtk"))
    assert e.value.status == 8
