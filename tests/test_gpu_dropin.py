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
                                  "bump_weno_explicit_fallback", "sod_movers1_single_efix_explicit",
                                  "cyl_movers2_efix_lts", "cyl_ricca2_lts", "bump_nwsc2_rk3"])
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


@pytest.mark.parametrize("name", ["cyl_roe2_lts", "sod_roe2_explicit"])
def test_lazy_copies_give_the_reference_results(name):
    """The same runs with the globals copied back at every 7th Update() only (and once when the
    harness loop returns): the reference's results bit for bit, Min_dt and Error every step."""
    import ctypes
    import os
    from oracle import refpy
    if not os.path.exists(refpy.DROPIN_LIB):
        pytest.skip("oracle/_ref/libcfdref_dropin.so not built (reference sources absent at build time)")
    case = CASES[name]
    g = load_golden(name)
    m = make_mesh(case)
    r = refpy.RefRun(m, ref_params(case), lib_path=refpy.DROPIN_LIB)
    r.L.refh_set_shim_sync.argtypes = [ctypes.c_int]
    r.L.refh_set_shim_sync.restype = ctypes.c_int
    assert r.L.refh_set_shim_sync(7) == 0
    r.set_state(g["U0"])
    n = r.iterate(case["steps"], case.get("t_end", 0.0))
    r.L.refh_set_shim_sync(1)
    assert n == int(g["iterations"][0])
    st = r.state()
    for k in ("U", "prim", "dt", "net_flux", "delU"):
        assert_bits_equal(st[k], g[k], name + ":" + k)
    assert_bits_equal(np.array([r.total_time()]), g["total_time"], "Total_Time")
    np.testing.assert_allclose(r.error(), g["error"], rtol=1e-12, atol=0)


def test_calculate_flux_for_all_faces_with_the_reference_dissipation():
    """The shim's Calculate_Flux_For_All_Faces (src/Net_Flux.cpp:7-43) with the reference's own
    ROE_2O as the callback, summed over every cell from zero, equals the net flux of the
    reference's Evaluate_Cell_Net_Flux_2O on the same state (the unmodified reference library)."""
    import ctypes
    import os
    from oracle import refpy
    if not os.path.exists(refpy.DROPIN_LIB):
        pytest.skip("oracle/_ref/libcfdref_dropin.so not built (reference sources absent at build time)")
    case = CASES["cyl_roe2_lts"]
    g = load_golden("cyl_roe2_lts")
    m = make_mesh(case)
    NP = m.n_physical
    want = []
    for lib in (refpy.REF_LIB, refpy.DROPIN_LIB):
        r = refpy.RefRun(m, ref_params(case), lib_path=lib)
        r.set_state(g["U0"])
        r.iterate(5)
        out = np.zeros((NP, 4))
        r.L.refh_net_flux_by_faces.argtypes = [ctypes.POINTER(ctypes.c_double)]
        r.L.refh_net_flux_by_faces.restype = None
        r.L.refh_net_flux_by_faces(out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        want.append(out)
    assert_bits_equal(want[1], want[0], "net flux by Calculate_Flux_For_All_Faces (drop-in vs reference)")


def test_lax_friedrichs_through_the_shim():
    """The shim's Lax_Fedrichs (src/Numerical_Method.cpp:459) in a reference process: the same U as
    the unmodified reference library."""
    import os
    from oracle import refpy
    if not os.path.exists(refpy.DROPIN_LIB):
        pytest.skip("oracle/_ref/libcfdref_dropin.so not built (reference sources absent at build time)")
    case = CASES["cyl_roe2_lts"]
    g = load_golden("lax_friedrichs_reference")
    m = make_mesh(case)
    r = refpy.RefRun(m, ref_params(case), lib_path=refpy.DROPIN_LIB)
    r.set_state(g["cyl_roe2_lts_U0"])
    r.L.refh_apply_bc()
    r.L.refh_net_flux()
    r.L.refh_lax_friedrichs()
    assert_bits_equal(r.state()["U"], g["cyl_roe2_lts_U"], "U after Lax_Fedrichs through the shim")


def test_reference_driver_throughput_on_the_half_cylinder(capsys):
    """The reference's own loop through the drop-in on the full 1024 x 512 half-cylinder O-grid
    (its ROE_2O + MinMod scheme with Runge_Kutta_Method and local dt, M = 3): cell-updates/s with
    the globals copied after every entry point and with lazy copies (once at the end of the loop).
    The figures are printed; the lazy form must be the faster one."""
    import ctypes
    import os
    import time
    from oracle import ogrid, refpy
    if not os.path.exists(refpy.DROPIN_LIB):
        pytest.skip("oracle/_ref/libcfdref_dropin.so not built (reference sources absent at build time)")
    params = {"CFL": 0.8, "Time_Accurate": 1, "Dissipation_Type": 3, "Is_Second_Order": 1, "Local_Time_Stepping": 1,
              "Inlet_Rho": 1.0, "Inlet_P": 1.0 / 1.4}
    r = ogrid.reference_half_cylinder(1024, 512, 1.0, 4.0, 1.005, params, lib_path=refpy.DROPIN_LIB)
    r.L.refh_set_shim_sync.argtypes = [ctypes.c_int]
    r.L.refh_set_shim_sync.restype = ctypes.c_int
    r.iterate(2)
    rates = {}
    for label, k, n in (("eager", 1, 10), ("lazy", 0, 100)):
        r.L.refh_set_shim_sync(k)
        t = time.perf_counter()
        r.iterate(n)
        rates[label] = r.NP * n / (time.perf_counter() - t)
    r.L.refh_set_shim_sync(1)
    with capsys.disabled():
        print("\ndrop-in throughput, reference driver on the 1024x512 O-grid: eager copies %.3e, lazy copies %.3e "
              "cell-updates/s" % (rates["eager"], rates["lazy"]))
    assert rates["lazy"] > rates["eager"]
