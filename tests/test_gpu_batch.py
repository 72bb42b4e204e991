"""Batched solves (cfd_batch_*): uneven ramp meshes run together in one union mesh with work
lists.  Each instance's state must equal the same mesh solved alone, bit for bit, also for
instances that stop early when their residual has dropped below the tolerance."""
import numpy as np
import pytest

import cfd_solver_withcuda_b200 as cb
from conftest import assert_bits_equal

pytestmark = pytest.mark.gpu
GAMMA = 1.4


def ramp_case(nx, ny, mach):
    m = cb.Mesh.ramp(nx, ny, 3.0, 1.0, 1.0, 15.0, open_top=True)
    rho, p = 1.0, 1.0 / GAMMA
    u = mach * np.sqrt(GAMMA * p / rho)
    NP = m.n_physical
    U = cb.conserved_from_primitive(np.full(NP, rho), np.full(NP, u), np.zeros(NP), np.full(NP, p))
    full = np.zeros((m.n_total, 4))
    full[:NP] = U
    full[m.boundary[:, 3]] = U[m.boundary[:, 1]]
    return m, full, (rho, u, 0.0, p)


def config(**kw):
    base = dict(dissipation_type=3, is_second_order=1, time_accurate=1, local_time_stepping=1, cfl=0.8,
                limiter=cb.LIM_VANLEER, muscl=cb.MUSCL_GRADIENT, integrator=cb.INT_SSPRK3,
                inlet_bc=cb.INLET_FIXED, reorder=0)
    base.update(kw)
    return cb.default_config(**base)


@pytest.mark.parametrize("precision", [cb.PREC_FP64, cb.PREC_FP32_FLUX])
def test_batch_instances_equal_single_solves(precision):
    specs = [(24, 12, 1.5), (40, 20, 2.2), (16, 8, 3.0), (32, 24, 2.6)]
    cases = [ramp_case(*sp) for sp in specs]
    b = cb.Batch([c[0] for c in cases], config(precision=precision), inflow=[c[2] for c in cases])
    b.upload_state([c[1] for c in cases])
    res = b.run(max_steps=60, tol=0.0, check_every=20)
    assert res["steps"] == 60
    assert res["cell_updates"] == 60 * sum(c[0].n_physical for c in cases)
    got = b.download_state()
    for (m, U0, q), Ub in zip(cases, got):
        rho, u, v, p = q
        s = cb.Solver(m, config(precision=precision, inlet_rho=rho, inlet_u=u, inlet_v=v, inlet_p=p))
        s.upload_state(U0)
        s.step(60)
        assert_bits_equal(Ub, s.download_U(), "instance %dx%d" % (m.n_physical, 0))


def test_batch_converged_instances_freeze():
    specs = [(16, 8, 2.0), (48, 16, 2.0)]
    cases = [ramp_case(*sp) for sp in specs]
    # MinMod: its residual falls to round-off on these ramps (Van Leer's stalls near 1e-3).
    b = cb.Batch([c[0] for c in cases], config(limiter=cb.LIM_MINMOD), inflow=[c[2] for c in cases])
    b.upload_state([c[1] for c in cases])
    res = b.run(max_steps=3000, tol=1e-6, check_every=25)
    sto = res["steps_to_tol"]
    assert sto[0] > 0 and sto[1] > 0, res
    assert np.all(res["res_ratio"] <= 1e-6)
    got = b.download_state()
    for (m, U0, q), Ub, k in zip(cases, got, sto):
        rho, u, v, p = q
        s = cb.Solver(m, config(limiter=cb.LIM_MINMOD, inlet_rho=rho, inlet_u=u, inlet_v=v, inlet_p=p))
        s.upload_state(U0)
        s.step(int(k))
        assert_bits_equal(Ub, s.download_U(), "frozen instance")
    assert res["cell_updates"] == sum(int(k) * c[0].n_physical for c, k in zip(cases, sto))
