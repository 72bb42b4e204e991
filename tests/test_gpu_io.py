"""Solution files written and read by the GPU context against the reference's Write_Solution and
its restart arithmetic (Initialize(const string &), src/Initialize.cpp:125-176)."""
import numpy as np
import pytest

import cfd_solver_withcuda_b200 as cb
from cases import CASES, make_mesh, ref_params, solver_config
from conftest import assert_bits_equal, load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["cyl_roe2_lts", "sod_roe2_rk3"])
def test_write_solution_matches_reference_bytes(name, tmp_path):
    from oracle import refpy
    if not refpy.ref_available():
        pytest.skip("oracle/_ref/libcfdref.so not built (reference sources absent at build time)")
    case = CASES[name]
    m = make_mesh(case)
    g = load_golden(name)
    r = refpy.RefRun(m, ref_params(case))
    r.set_state(g["U0"])
    r.iterate(7)
    a = tmp_path / "ref.txt"
    r.L.refh_write_solution(str(a).encode())
    s = cb.Solver(m, solver_config(case))
    s.upload_state(g["U0"])
    s.step(7)
    b = tmp_path / "mine.txt"
    s.write_solution(b)
    assert a.read_bytes() == b.read_bytes()


def test_read_solution_restart_state(tmp_path):
    """Physical rows from a written file: U = (rho, rho u, rho v, p/(gamma-1) + rho |V|^2 / 2) of the
    file's values (six significant digits), ghost rows untouched, iteration count restored; a
    mismatched cell count is refused."""
    case = CASES["cyl_roe2_lts"]
    m = make_mesh(case)
    g = load_golden("cyl_roe2_lts")
    s = cb.Solver(m, solver_config(case))
    s.upload_state(g["U0"])
    s.step(9)
    path = tmp_path / "sol.txt"
    s.write_solution(path)
    rows = np.loadtxt(path, skiprows=3)
    rho, p, u, v = rows[:, 2], rows[:, 3], rows[:, 5], rows[:, 6]
    want = np.stack([rho, rho * u, rho * v, (p / (1.4 - 1.0)) + rho * (0.5 * (u * u + v * v))], axis=1)
    t = cb.Solver(m, solver_config(case))
    t.upload_state(g["U0"])
    ghosts_before = t.download_U()[m.n_physical:].copy()
    t.read_solution(path)
    U = t.download_U()
    assert_bits_equal(U[:m.n_physical], want, "restart U")
    assert_bits_equal(U[m.n_physical:], ghosts_before, "ghost rows")
    assert t.step(0).iterations == 9
    other = cb.Solver(make_mesh(CASES["sod_roe2_rk3"]), solver_config(CASES["sod_roe2_rk3"]))
    with pytest.raises(cb.CfdError) as e:
        other.read_solution(path)
    assert e.value.status == 7
