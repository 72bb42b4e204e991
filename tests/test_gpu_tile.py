"""The tile form (reorder = 4 on a structured block: one thread block per 32 x 8 tile does the
gradients, face fluxes, gather and stage update of its cells with the states of two rings around it
in shared memory) against the C restatement and against the three-kernel form, bit for bit, in both
of its variants: tile_stage 1 (loads inside the phases) and 2 (the TMA form: tensor loads of the
state rows and face records, cp.async of the stage inputs, all issued at block start)."""
import numpy as np
import pytest

import cfd_solver_withcuda_b200 as cb
from cases import CASES, initial_state, make_mesh, oracle_params, solver_config
from conftest import assert_bits_equal

pytestmark = pytest.mark.gpu

GRAD = dict(muscl=cb.MUSCL_GRADIENT, is_second_order=1, time_accurate=1, local_time_stepping=1)
TILE_FORMS = {
    "roe_vanleer_ssp": dict(GRAD, dissipation_type=cb.DISS_ROE, limiter=cb.LIM_VANLEER, integrator=cb.INT_SSPRK3),
    "roe_minmod_ssp": dict(GRAD, dissipation_type=cb.DISS_ROE, limiter=cb.LIM_MINMOD, integrator=cb.INT_SSPRK3),
    "roe_vanleer_fixes_ssp": dict(GRAD, dissipation_type=cb.DISS_ROE, limiter=cb.LIM_VANLEER, integrator=cb.INT_SSPRK3,
                                  entropy_fix_linear=0.4, shock_fix=0.2),
    "hllc_minmod_ssp": dict(GRAD, dissipation_type=cb.DISS_HLLC, limiter=cb.LIM_MINMOD, integrator=cb.INT_SSPRK3),
    "ausm_vanalbada_ssp": dict(GRAD, dissipation_type=cb.DISS_AUSM, limiter=cb.LIM_VANALBADA,
                               integrator=cb.INT_SSPRK3),
    "ausm_gpu_superbee_ssp": dict(GRAD, dissipation_type=cb.DISS_AUSM_GPU, limiter=cb.LIM_SUPERBEE,
                                  integrator=cb.INT_SSPRK3),
    "roe_vanleer_rk3_gpu_ref": dict(GRAD, dissipation_type=cb.DISS_ROE, limiter=cb.LIM_VANLEER,
                                    integrator=cb.INT_RK3_GPU_REF),
    "roe_vanleer_fp32": dict(GRAD, dissipation_type=cb.DISS_ROE, limiter=cb.LIM_VANLEER, integrator=cb.INT_SSPRK3,
                             precision=cb.PREC_FP32_FLUX),
    "hllc_minmod_fp32": dict(GRAD, dissipation_type=cb.DISS_HLLC, limiter=cb.LIM_MINMOD, integrator=cb.INT_SSPRK3,
                             precision=cb.PREC_FP32_FLUX),
    "roe_minmod_fixes_fp32": dict(GRAD, dissipation_type=cb.DISS_ROE, limiter=cb.LIM_MINMOD, integrator=cb.INT_SSPRK3,
                                  precision=cb.PREC_FP32_FLUX, shock_fix=0.1),
}

# Structured meshes: the half-cylinder O-grid (48 x 24: a partial tile in i), the ramp (52 x 18:
# partial tiles in both directions), the Sod box (100 x 4: thinner than a tile), and a box with
# the reference's subsonic inlet and the subsonic exit whose ghosts no boundary condition writes.
SUBSONIC_BOX = dict(mesh=("box", 70, 13, 0.0, 2.0, 0.0, 1.0), ic="pulse", mach=0.5, dissipation_type=3,
                    is_second_order=1, time_accurate=1, cfl=0.5, inlet_rho=1.0, inlet_p=1.0 / 1.4, inlet_bc=1,
                    exit_bc=1)
BASES = {"cyl": CASES["cyl_roe2_lts"], "ramp": dict(CASES["ramp_roe1_explicit"], time_accurate=1),
         "sod": CASES["sod_roe2_rk3"], "subsonic_box": SUBSONIC_BOX}


def check_state(a, b, what, keys=("U", "prim", "dt", "net_flux", "delU")):
    for k in keys:
        assert_bits_equal(a[k], b[k], what + ":" + k)


def tile_launches(s, steps):
    """Runs `steps` pseudo-steps with per-launch timing on and returns the tile-kernel launches."""
    s.set_option("profile", 1)
    s.step(steps)
    s.set_option("profile", 0)
    return s.kernel_time("tile")[1]


@pytest.mark.parametrize("variant", [1, 2, 3, 4])
@pytest.mark.parametrize("base", sorted(BASES))
@pytest.mark.parametrize("form", sorted(TILE_FORMS))
def test_tile_form_matches_oracle(form, base, variant, oracle_lib):
    case = BASES[base]
    over = TILE_FORMS[form]
    m = make_mesh(case)
    U0 = initial_state(case, m)
    steps = 24
    s = cb.Solver(m, solver_config(case, reorder=4, **over))
    s.set_option("tile_stage", variant)
    s.upload_state(U0)
    assert tile_launches(s, 4) == 4 * 3
    s.step(steps - 4)
    o = oracle_lib.OracleRun(m, **oracle_params(case, **over))
    o.set_state(U0)
    o.iterate(steps)
    check_state(s.download(), o.state(), form)
    assert s.info.total_time == o.total_time()
    np.testing.assert_allclose(np.array(s.info.error[:]), o.error(), rtol=1e-12, atol=0)


@pytest.mark.parametrize("form", ["roe_vanleer_ssp", "hllc_minmod_fp32", "roe_vanleer_rk3_gpu_ref"])
def test_tile_form_equals_three_kernel_form(form):
    """Same context configuration, tile form on and off, with and without graph replay."""
    case = BASES["cyl"]
    m = make_mesh(case)
    U0 = initial_state(case, m)
    outs = []
    for tile, graph in ((1, 1), (0, 1), (1, 0), (2, 1), (2, 0), (3, 1), (4, 1), (4, 0)):
        s = cb.Solver(m, solver_config(case, reorder=4, **TILE_FORMS[form]))
        s.set_option("tile_stage", tile)
        s.set_option("use_graph", graph)
        s.upload_state(U0)
        s.step(15)
        outs.append((s.download(), np.array(s.info.error[:])))
    for o, err in outs[1:]:
        check_state(o, outs[0][0], form)
        np.testing.assert_allclose(err, outs[0][1], rtol=1e-12, atol=0)


@pytest.mark.parametrize("variant", [1, 2, 3, 4])
def test_tile_form_entry_points_interleave(variant, oracle_lib):
    """Entry points called between tile steps (an upload, the reference's one-call stages) see and
    leave a consistent state: the tile form starts every step from the current rows."""
    case = BASES["cyl"]
    over = TILE_FORMS["roe_minmod_ssp"]
    m = make_mesh(case)
    U0 = initial_state(case, m)
    s = cb.Solver(m, solver_config(case, reorder=4, **over))
    s.set_option("tile_stage", variant)
    o = oracle_lib.OracleRun(m, **oracle_params(case, **over))
    s.upload_state(U0)
    o.set_state(U0)
    s.step(3)
    o.iterate(3)
    U1 = s.download()["U"]
    s.upload_state(U1)
    o.set_state(U1)
    s.step(5)
    o.iterate(5)
    check_state(s.download(), o.state(), "after re-upload")


def test_reorder4_refuses_mixed_mesh():
    case = CASES["bump_roe2_rk3"]
    m = make_mesh(case)
    with pytest.raises(cb.CfdError):
        cb.Solver(m, solver_config(case, reorder=4, **TILE_FORMS["roe_vanleer_ssp"]))


def test_tile_option_needs_block():
    case = BASES["cyl"]
    m = make_mesh(case)
    s = cb.Solver(m, solver_config(case, reorder=1, **TILE_FORMS["roe_vanleer_ssp"]))
    for v in (1, 2, 3, 4):
        with pytest.raises(cb.CfdError):
            s.set_option("tile_stage", v)
    s.set_option("tile_stage", 0)
    t = cb.Solver(m, solver_config(case, reorder=4, **TILE_FORMS["roe_vanleer_ssp"]))
    with pytest.raises(cb.CfdError):
        t.set_option("tile_stage", 5)


def test_tile_tma_form_on_the_benchmark_block(oracle_lib):
    """The TMA form on a 256 x 96 O-grid (8 x 12 tiles, every tile interior or on one rim) with the
    benchmark's scheme, 30 steps, bit for bit against the C restatement."""
    m = cb.Mesh.half_cylinder(256, 96, 1.0, 4.0, 1.005)
    NP = m.n_physical
    rho, p = 1.0, 1.0 / 1.4
    u = 3.0 * np.sqrt(1.4 * p / rho)
    U = cb.conserved_from_primitive(np.full(NP, rho), np.full(NP, u), np.zeros(NP), np.full(NP, p))
    U0 = np.zeros((m.n_total, 4))
    U0[:NP] = U
    U0[m.boundary[:, 3]] = U[m.boundary[:, 1]]
    kw = dict(dissipation_type=3, is_second_order=1, time_accurate=1, local_time_stepping=1, cfl=0.8, limiter=2,
              muscl=1, integrator=2, inlet_rho=rho, inlet_p=p, inlet_bc=3, inlet_u=u, inlet_v=0.0)
    s = cb.Solver(m, cb.default_config(device=0, reorder=4, **kw))
    s.set_option("tile_stage", 2)
    s.upload_state(U0)
    assert tile_launches(s, 3) == 9
    s.step(27)
    o = oracle_lib.OracleRun(m, **kw)
    o.set_state(U0)
    o.iterate(30)
    check_state(s.download(), o.state(), "tma")
