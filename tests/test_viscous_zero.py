"""Why the path has no viscous flux: the reference has no working viscous residual to replace.

(1) Its co-volume set-up cannot complete.  Construct_Co_Volumes
(src/Co_Volume_Grid_Computations.cpp:30-33) assigns the cell's whole Cell_Vertices vector to each
of the four corner points o, a, b, c, so every co-volume diagonal it forms is the zero vector and
Evaluate_Cross_Product (src/Grid_Computations.cpp:834-844) prints "Check Area 0" and calls exit(0)
on the first quad cell.  Form_Cells runs this for every cell when the wall is viscous
(src/Grid_Computations.cpp:367-375), so a viscous run of the reference ends there.
(2) Past that point the result would still be zero: the co-volume pushed is a value-initialised
Cell whose empty Face_Areas, Face_Normals and Cell_Areas are resized to zeros and whose Inv_Area is
never set (src/Co_Volume_Grid_Computations.cpp:96-118), and Calculate_Gradient_On_Face
(src/Grid_Refine_Functions.cpp:266-416) is a sum over those faces times that inverse area.

The test runs the reference's own code (oracle/_ref, built from its sources) in a child process,
on a flow with developed gradients, and checks that the viscous evaluation terminates the process
in the co-volume set-up, on the first cell, before any viscous flux is formed."""
import os
import subprocess
import sys
import textwrap

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = textwrap.dedent("""
    import ctypes, sys
    sys.path.insert(0, %r)
    import numpy as np
    import cfd_solver_withcuda_b200 as cb
    from oracle import refpy
    m = cb.Mesh.half_cylinder(32, 16, 1.0, 4.0, 1.04)
    NP = m.n_physical
    rho, p = 1.0, 1.0 / 1.4
    u = 3.0 * np.sqrt(1.4 * p / rho)
    U = cb.conserved_from_primitive(np.full(NP, rho), np.full(NP, u), np.zeros(NP), np.full(NP, p))
    U0 = np.zeros((m.n_total, 4)); U0[:NP] = U; U0[m.boundary[:, 3]] = U[m.boundary[:, 1]]
    r = refpy.RefRun(m, {"CFL": 0.5, "Time_Accurate": 1, "Dissipation_Type": 3, "Is_Second_Order": 0,
                         "Inlet_Rho": rho, "Inlet_P": p})
    r.set_state(U0)
    r.iterate(30)
    st = r.state()
    print("GRADIENTS", float(np.ptp(st["prim"][:NP, 0])), float(np.ptp(st["prim"][:NP, 4])), flush=True)
    L = r.L
    dp = ctypes.POINTER(ctypes.c_double)
    L.refh_viscous_flux.argtypes = [ctypes.c_double, ctypes.c_double, dp, dp]
    L.refh_viscous_flux.restype = None
    flux = np.full((NP, 4), np.nan)
    covol = np.full(3, np.nan)
    L.refh_viscous_flux(0.01, 2.5, flux.ctypes.data_as(dp), covol.ctypes.data_as(dp))
    print("VISCOUS_FLUX_FORMED", np.count_nonzero(flux), covol.tolist(), flush=True)
""") % ROOT


def test_reference_viscous_path_terminates_in_co_volume_setup():
    from oracle import refpy
    if not refpy.ref_available():
        pytest.skip("oracle/_ref/libcfdref.so was not built (reference sources absent)")
    r = subprocess.run([sys.executable, "-c", CHILD], capture_output=True, text=True, timeout=300)
    out = r.stdout
    grad = [l for l in out.splitlines() if l.startswith("GRADIENTS")]
    assert grad, out + r.stderr
    d_rho, d_p = map(float, grad[0].split()[1:])
    assert d_rho > 0.5 and d_p > 0.5  # a bow shock has formed (density and pressure ranges)
    assert "In Evaluating Cross Product..... Check Area\t0" in out, out
    assert "VISCOUS_FLUX_FORMED" not in out
    assert r.returncode == 0  # the reference's exit(0)
