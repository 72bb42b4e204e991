"""The one-kernel patch stage (reorder = 3: recursive-bisection patches of 128 cells, one thread
block per patch doing gradients, face fluxes, gather and stage update) against the C restatement
and against the three-kernel form, bit for bit."""
import numpy as np
import pytest

import cfd_solver_withcuda_b200 as cb
from cases import CASES, initial_state, make_mesh, oracle_params, solver_config
from conftest import assert_bits_equal

pytestmark = pytest.mark.gpu

GRAD = dict(muscl=cb.MUSCL_GRADIENT, is_second_order=1, time_accurate=1, local_time_stepping=1)
PATCH_FORMS = {
    "roe_vanleer_ssp": dict(GRAD, dissipation_type=cb.DISS_ROE, limiter=cb.LIM_VANLEER, integrator=cb.INT_SSPRK3),
    "roe_minmod_ssp": dict(GRAD, dissipation_type=cb.DISS_ROE, limiter=cb.LIM_MINMOD, integrator=cb.INT_SSPRK3),
    "hllc_minmod_ssp": dict(GRAD, dissipation_type=cb.DISS_HLLC, limiter=cb.LIM_MINMOD, integrator=cb.INT_SSPRK3),
    "ausm_vanalbada_ssp": dict(GRAD, dissipation_type=cb.DISS_AUSM, limiter=cb.LIM_VANALBADA,
                               integrator=cb.INT_SSPRK3),
    "ausm_gpu_superbee_ssp": dict(GRAD, dissipation_type=cb.DISS_AUSM_GPU, limiter=cb.LIM_SUPERBEE,
                                  integrator=cb.INT_SSPRK3),
    "roe_vanleer_rk4": dict(GRAD, dissipation_type=cb.DISS_ROE, limiter=cb.LIM_VANLEER, integrator=cb.INT_RK4),
    "roe_minmod_rk4_gpu_ref": dict(GRAD, dissipation_type=cb.DISS_ROE, limiter=cb.LIM_MINMOD,
                                   integrator=cb.INT_RK4_GPU_REF),
    "roe_vanleer_rk3_gpu_ref": dict(GRAD, dissipation_type=cb.DISS_ROE, limiter=cb.LIM_VANLEER,
                                    integrator=cb.INT_RK3_GPU_REF),
}
STAGES = {cb.INT_SSPRK3: 3, cb.INT_RK4: 4, cb.INT_RK4_GPU_REF: 4, cb.INT_RK3_GPU_REF: 3}


def check_state(a, b, what, keys=("U", "prim", "dt", "net_flux", "delU")):
    for k in keys:
        assert_bits_equal(a[k], b[k], what + ":" + k)


def patch_launches(s, steps):
    """Runs `steps` pseudo-steps with per-launch timing on and returns the patch-kernel launches."""
    s.set_option("profile", 1)
    s.step(steps)
    s.set_option("profile", 0)
    return s.kernel_time("patch")[1]


# cyl: quads with wall, supersonic inlet and exit ghosts; bump: mixed triangles and quads;
# bump_llf1_subsonic: the reference subsonic inlet and the subsonic exit, whose ghosts no BC writes.
@pytest.mark.parametrize("base", ["cyl_roe2_lts", "bump_roe2_rk3", "bump_llf1_subsonic"])
@pytest.mark.parametrize("form", sorted(PATCH_FORMS))
def test_patch_form_matches_oracle(form, base, oracle_lib):
    case = CASES[base]
    over = PATCH_FORMS[form]
    m = make_mesh(case)
    U0 = initial_state(case, m)
    steps = 24
    s = cb.Solver(m, solver_config(case, reorder=3, **over))
    s.set_option("patch_stage", 1)
    s.upload_state(U0)
    assert patch_launches(s, 4) == 4 * STAGES[over["integrator"]]
    s.step(steps - 4)
    o = oracle_lib.OracleRun(m, **oracle_params(case, **over))
    o.set_state(U0)
    o.iterate(steps)
    check_state(s.download(), o.state(), form)
    assert s.info.total_time == o.total_time()
    assert s.info.iterations == steps


def halfcyl(nt, nr):
    m = cb.Mesh.half_cylinder(nt, nr, 1.0, 4.0, 1.005)
    case = dict(CASES["cyl_roe2_lts"])
    return m, case, initial_state(case, m)


@pytest.mark.parametrize("form", ["roe_vanleer_ssp", "hllc_minmod_ssp", "roe_vanleer_rk4"])
def test_patch_form_equals_three_kernel_form(form):
    """256 x 128 O-grid (256 patches): patch form, the three-kernel form on the same numbering and
    on RCM numbering give the same fields bit for bit; the norms are tree reductions over
    different block partitions, equal within 1e-12; t_end ends all three on the same step."""
    m, case, U0 = halfcyl(256, 128)
    over = PATCH_FORMS[form]
    runs = []
    for reorder, patch in ((3, 1), (3, 0), (1, 1)):
        s = cb.Solver(m, solver_config(case, reorder=reorder, **over))
        s.set_option("patch_stage", patch)
        s.upload_state(U0)
        s.step(30)
        t_mid = s.info.total_time
        s.step(1000, t_mid * 1.5)
        runs.append((s.download(), s.info.iterations, s.info.total_time, np.array(s.info.res_l2[:]),
                     np.array(s.info.error[:])))
    ref = runs[0]
    assert 30 < ref[1] < 1030
    for st, it, t, res, err in runs[1:]:
        check_state(st, ref[0], form)
        assert it == ref[1] and t == ref[2]
        np.testing.assert_allclose(res, ref[3], rtol=1e-12)
        np.testing.assert_allclose(err, ref[4], rtol=1e-12)


def test_patch_option_and_autotune():
    """With patch tables the autotuner adds the patch candidates; tuning leaves the state and
    the later bits unchanged."""
    m, case, U0 = halfcyl(96, 48)
    cfg = solver_config(case, reorder=3, **PATCH_FORMS["roe_vanleer_ssp"])
    a = cb.Solver(m, cfg)
    a.upload_state(U0)
    a.step(3)
    before = a.download()
    report = a.autotune(steps=5)
    assert report.count("ms/step") == 22 and report.count("patch_stage=1") == 2, report
    check_state(a.download(), before, "after autotune")
    a.step(10)
    b = cb.Solver(m, cfg)
    b.set_option("patch_stage", 0)
    b.upload_state(U0)
    b.step(13)
    check_state(a.download(), b.download(), "tuned vs three-kernel")


def test_entry_points_after_patch_steps(oracle_lib):
    """After patch-form pseudo-steps the reference entry points (boundary conditions, net flux,
    Runge_Kutta_Method, Estimate_Error, Update) continue from the same state as the oracle."""
    case = CASES["cyl_roe2_lts"]
    over = PATCH_FORMS["roe_minmod_ssp"]
    m = make_mesh(case)
    U0 = initial_state(case, m)
    s = cb.Solver(m, solver_config(case, reorder=3, **over))
    s.set_option("patch_stage", 1)
    s.upload_state(U0)
    s.step(10)
    s.Apply_Boundary_Conditions()
    s.Runge_Kutta_Method()
    s.Estimate_Error()
    s.Update()
    s.step(5)
    o = oracle_lib.OracleRun(m, **oracle_params(case, **over))
    o.set_state(U0)
    o.iterate(10)
    o.apply_bc()
    o.rk()
    o.estimate_error()
    o.update()
    o.iterate(5)
    check_state(s.download(), o.state(), "mixed")
