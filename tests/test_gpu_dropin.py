"""The drop-in: the reference's own solver loop (src/Solver.cpp:94-125, replayed by the oracle
harness) with cfd_solver_withcuda_b200/dropin/b200_shim.cpp linked in place of
Numerical_Method.cpp, Net_Flux.cpp and Error_Estimate_Update.cpp, so that Runge_Kutta_Method /
Explicit_Method / Estimate_Error / Update run on the GPU through libcfd_b200.so.  Its results must
be those of the unmodified reference (golden fixtures) bit for bit."""
import numpy as np
import pytest

from cases import CASES, make_mesh, ref_params
from conftest import assert_bits_equal, load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["sod_roe1_rk3", "sod_roe2_rk3", "sod_llf1_rk3", "sod_roe2_explicit", "cyl_roe2_lts",
                                  "bump_roe2_rk3", "ramp_roe1_explicit", "pulse_weno_rk3", "sod_weno_char_rk3",
                                  "bump_weno_explicit_fallback"])
def test_reference_driver_on_the_gpu_path(name):
    from oracle import refpy
    import os
    if not os.path.exists(refpy.DROPIN_LIB):
        pytest.skip("oracle/_ref/libcfdref_dropin.so not built (reference sources absent at build time)")
    case = CASES[name]
    g = load_golden(name)
    m = make_mesh(case)
    r = refpy.RefRun(m, ref_params(case), lib_path=refpy.DROPIN_LIB)
    r.set_state(g["U0"])
    n = r.iterate(case["steps"], case.get("t_end", 0.0))
    assert n == int(g["iterations"][0])
    st = r.state()
    for k in ("U", "prim", "dt", "net_flux", "delU"):
        assert_bits_equal(st[k], g[k], name + ":" + k)
    assert_bits_equal(np.array([r.total_time()]), g["total_time"], "Total_Time")
    np.testing.assert_allclose(r.error(), g["error"], rtol=1e-12, atol=0)
