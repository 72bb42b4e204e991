"""Edge sizes: meshes of one to a few cells (one partially filled thread block, cells whose every
neighbour is a ghost, a face list shorter than a warp) in the reference's per-cell forms and the
face-based forms, every field bit for bit against the C restatement after a few steps, with the
default launch options and with every option set the tuner may pick."""
import numpy as np
import pytest

import cfd_solver_withcuda_b200 as cb
from conftest import assert_bits_equal

pytestmark = pytest.mark.gpu

GAMMA = 1.4
MESHES = [(1, 1), (2, 1), (1, 3), (3, 2), (5, 1), (7, 5)]
FORMS = {
    "reference_roe2_rk3": dict(dissipation_type=3, is_second_order=1, time_accurate=1, cfl=0.5),
    "reference_roe1_explicit": dict(dissipation_type=3, is_second_order=0, time_accurate=0, cfl=0.4),
    "reference_llf1_rk3": dict(dissipation_type=1, is_second_order=0, time_accurate=1, cfl=0.4),
    "muscl_vanleer_prim_ssprk3_lts": dict(dissipation_type=3, is_second_order=1, time_accurate=1,
                                          local_time_stepping=1, cfl=0.8, muscl=1, limiter=2,
                                          reconstruct_primitive=1, integrator=2),
    "muscl_fp32_flux_ssprk3_lts": dict(dissipation_type=3, is_second_order=1, time_accurate=1,
                                       local_time_stepping=1, cfl=0.8, muscl=1, limiter=2,
                                       reconstruct_primitive=1, integrator=2, precision=1),
    "muscl_hllc_minmod_rk3": dict(dissipation_type=7, is_second_order=1, time_accurate=1, cfl=0.5, muscl=1,
                                  limiter=1, integrator=2),
}
STEPS = 6


def state(m, seed):
    """A smooth, positive, non-uniform state (M about 1.5 along x) with ghosts copied from their
    owners, so that every face sees a jump."""
    rng = np.random.default_rng(seed)
    NP = m.n_physical
    rho = 1.0 + 0.2 * rng.random(NP)
    p = (1.0 + 0.3 * rng.random(NP)) / GAMMA
    u = 1.5 * np.sqrt(GAMMA * p / rho) * (1.0 + 0.1 * rng.random(NP))
    v = 0.1 * (rng.random(NP) - 0.5)
    U = cb.conserved_from_primitive(rho, u, v, p)
    full = np.zeros((m.n_total, 4))
    full[:NP] = U
    full[m.boundary[:, 3]] = U[m.boundary[:, 1]]
    return full


def params(form):
    kw = dict(FORMS[form])
    kw.update(inlet_rho=1.0, inlet_p=1.0 / GAMMA)
    return kw


def run_gpu(m, U0, form, reorder, opts=None):
    s = cb.Solver(m, cb.default_config(reorder=reorder, **params(form)))
    for k, v in (opts or {}).items():
        s.set_option(k, v)
    s.upload_state(U0)
    s.step(STEPS)
    out = s.download()
    t = s.info.total_time
    s.close()
    return out, t


@pytest.mark.parametrize("reorder", [0, 1])
@pytest.mark.parametrize("form", sorted(FORMS))
@pytest.mark.parametrize("nx,ny", MESHES)
def test_small_mesh_matches_oracle(nx, ny, form, reorder, oracle_lib):
    m = cb.Mesh.box(nx, ny, 0.0, 1.0, 0.0, 0.5)
    U0 = state(m, nx * 100 + ny)
    out, t = run_gpu(m, U0, form, reorder)
    o = oracle_lib.OracleRun(m, **params(form))
    o.set_state(U0)
    o.iterate(STEPS)
    ref = o.state()
    for k in ("U", "prim", "dt", "net_flux", "delU"):
        assert_bits_equal(out[k], ref[k], "%s %dx%d %s" % (form, nx, ny, k))
    assert t == o.total_time()


@pytest.mark.parametrize("form", sorted(FORMS))
@pytest.mark.parametrize("nx,ny", [(1, 1), (3, 2)])
def test_small_mesh_tuned_options_keep_bits(nx, ny, form):
    """The tuner's choice on a mesh smaller than one thread block gives the default's bits."""
    m = cb.Mesh.box(nx, ny, 0.0, 1.0, 0.0, 0.5)
    U0 = state(m, 7)
    base, tb = run_gpu(m, U0, form, 1)
    s = cb.Solver(m, cb.default_config(reorder=1, **params(form)))
    s.upload_state(U0)
    report = s.autotune(steps=2)
    s.upload_state(U0)
    s.step(STEPS)
    out = s.download()
    assert s.info.total_time == tb
    s.close()
    for k in ("U", "prim", "dt", "net_flux", "delU"):
        assert_bits_equal(out[k], base[k], "%s tuned (%s) %s" % (form, report, k))
