"""The Python module CFD_Solver (cfd_solver_withcuda_b200/pybind/cfd_solver_module.cpp): the
reference wrapper's interface (Python_Wrapper/Euler_Python_Wrapper.cpp:92-159) over the C ABI.
On CPU: it loads and has the reference's function names.  On the GPU: the reference's driver
sequence through it gives the same bits as the ctypes binding, and Inviscid_Solver writes the
reference's files."""
import os

import numpy as np
import pytest

import cfd_solver_withcuda_b200 as cb
from cfd_solver_withcuda_b200 import build

REFERENCE_NAMES = ["readJSON", "testCase", "ReadGrid", "FormCells", "ConstructGhostCells", "Inviscid_Solver",
                   "Explicit_Method", "Runge_Kutta_Method", "Evaluate_Time_Step", "Inviscid_Time_Step",
                   "get_NoPhysical_Cells", "get_Min_dt", "get_Max_dt", "Apply_Boundary_Conditions",
                   "Estimate_Error", "Update", "Set_DelU"]


def _module():
    if not os.path.exists(build.pybind_path()):
        pytest.skip("CFD_Solver module not built (pybind11 absent at build time)")
    import importlib
    return importlib.import_module("cfd_solver_withcuda_b200.CFD_Solver")


def test_module_has_the_reference_entry_points():
    m = _module()
    missing = [n for n in REFERENCE_NAMES if not hasattr(m, n)]
    assert not missing, missing


def _config(tmp_path, **over):
    solver = {"Dissipation_Type": 3, "Is_Second_Order": True, "Time_Accurate": True, "Local_Time_Stepping": True}
    solver.update(over)
    import json
    cfg = {"Simulation": {"CFL": 0.5, "Total_Iterations": 2500},
           "Solver": solver,
           "BoundaryConditions": {"Is_Inlet_SubSonic": False, "Inlet_Rho": 1.0, "Inlet_P": 1.0}}
    p = tmp_path / "Solver_Config.json"
    p.write_text(json.dumps(cfg))
    return str(p)


@pytest.mark.gpu
def test_reference_sequence_matches_the_ctypes_binding(tmp_path):
    """Sod shock tube on a 100 x 4 box (a box domain, where the VTK reader's bounding-box boundary
    classification is the generator's), the reference's ROE_2O with its Runge_Kutta_Method."""
    M = _module()
    mesh = cb.Mesh.box(100, 4, 0.0, 1.0, 0.0, 0.01)
    grid = str(tmp_path / "grid.vtk")
    mesh.write_vtk(grid)
    cfgp = _config(tmp_path, Local_Time_Stepping=False)
    M.reset()
    M.readJSON(cfgp)
    M.testCase(1)
    assert M.ReadGrid(grid)
    M.ConstructGhostCells()
    assert M.FormCells()
    NP = M.get_NoPhysical_Cells()
    assert NP == mesh.n_physical
    xc = mesh.centers[:NP, 0]
    left = xc < 0.5
    U = cb.conserved_from_primitive(np.where(left, 1.0, 0.125), 0 * xc, 0 * xc, np.where(left, 1.0, 0.1))
    M.Set_State(U)
    s = cb.Solver(mesh, cb.read_config_json(cfgp, reorder=1))
    s.upload_state(U)
    for _ in range(5):
        for obj in (M, s):
            obj.Apply_Boundary_Conditions()
            obj.Runge_Kutta_Method()
            obj.Estimate_Error()
            obj.Update()
    want = s.download()
    assert np.array_equal(M.get_U().view(np.int64), want["U"].view(np.int64))
    assert np.array_equal(M.get_Primitive().view(np.int64), want["prim"].view(np.int64))
    assert M.get_Min_dt() == s.get_Min_dt()
    assert M.get_Max_dt() == float(want["dt"].max())
    # Set_DelU then Update: U += dU on the physical rows.
    dU = np.full((NP, 4), 1e-6)
    U0 = M.get_U()
    M.Set_DelU(dU.ravel())
    M.Update()
    np.testing.assert_array_equal(M.get_U()[:NP], U0[:NP] + dU)
    # The solver loop writes the error history and the solution file.
    M.Set_State(U)
    err, sol = str(tmp_path / "Error.txt"), str(tmp_path / "Solution.txt")
    assert M.Inviscid_Solver(err, sol)
    lines = open(err).read().splitlines()
    assert len(lines) == 1 + 3  # header + one line per 1000 iterations (2500 in 3 chunks)
    assert int(open(sol).read().splitlines()[1]) == NP
    M.reset()
