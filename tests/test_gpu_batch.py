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


@pytest.mark.parametrize("minb", [0, 4, 6, 8])
@pytest.mark.parametrize("precision", [cb.PREC_FP64, cb.PREC_FP32_FLUX])
def test_persistent_batch_equals_three_kernel_batch(precision, minb):
    """The persistent form (one cooperative launch per RK stage over the (instance, block) work
    lists, one CUDA graph per stage) gives every instance the bits of the three-kernel form, also
    when instances freeze at the tolerance in the middle of the run, for every register budget of
    the persistent kernel."""
    specs = [(24, 12, 1.5), (64, 32, 2.2), (16, 8, 3.0), (40, 24, 2.6), (12, 6, 2.0)]
    cases = [ramp_case(*sp) for sp in specs]
    out = []
    for persistent in (0, 1):
        b = cb.Batch([c[0] for c in cases], config(precision=precision, limiter=cb.LIM_MINMOD),
                     inflow=[c[2] for c in cases])
        b.set_option("persistent", persistent)
        b.set_option("persist_minb", minb)
        b.upload_state([c[1] for c in cases])
        res = b.run(max_steps=1500, tol=1e-4, check_every=50)
        out.append((res, b.download_state()))
        b.close()
    (r0, u0), (r1, u1) = out
    assert np.array_equal(r0["steps_to_tol"], r1["steps_to_tol"]), (r0["steps_to_tol"], r1["steps_to_tol"])
    assert (r0["steps_to_tol"] > 0).any()
    assert np.array_equal(r0["res_ratio"].view(np.int64), r1["res_ratio"].view(np.int64))
    for a, b_ in zip(u0, u1):
        assert_bits_equal(b_, a, "persistent vs three-kernel instance")


def test_persistent_single_solve_equals_default():
    """The persistent form on a single context (no work lists: the phases walk all rows, faces and
    cells) against the default kernels, on the half-cylinder O-grid with the benchmark scheme."""
    m = cb.Mesh.half_cylinder(64, 32, 1.0, 4.0, 1.04)
    NP = m.n_physical
    rho, p = 1.0, 1.0 / GAMMA
    u = 3.0 * np.sqrt(GAMMA * p / rho)
    U = cb.conserved_from_primitive(np.full(NP, rho), np.full(NP, u), np.zeros(NP), np.full(NP, p))
    U0 = np.zeros((m.n_total, 4))
    U0[:NP] = U
    U0[m.boundary[:, 3]] = U[m.boundary[:, 1]]
    got = []
    for persistent in (0, 1):
        s = cb.Solver(m, config(inlet_rho=rho, inlet_u=u, inlet_v=0.0, inlet_p=p, entropy_fix_linear=0.4, reorder=3))
        s.set_option("persistent", persistent)
        s.upload_state(U0)
        s.step(200)
        got.append(s.download())
        s.close()
    for k in ("U", "prim", "dt", "net_flux"):
        assert_bits_equal(got[1][k], got[0][k], "persistent single solve: " + k)


def test_persistent_barrier_wait_runs_out_with_a_status():
    """The bounded grid barrier: with one arrival that never comes, every wait runs out after its
    cycle limit, the step reports CFD_ERR_TIMEOUT, and the device stays usable (a fresh context
    then runs normally)."""
    m, U0, q = ramp_case(24, 12, 2.0)
    rho, u, v, p = q
    s = cb.Solver(m, config(inlet_rho=rho, inlet_u=u, inlet_v=v, inlet_p=p))
    s.set_option("persistent", 1)
    s.set_option("barrier_timeout_test", 1)
    s.upload_state(U0)
    with pytest.raises(cb.CfdError) as e:
        s.step(2)
    assert e.value.status == cb.CFD_ERR_TIMEOUT
    s.close()
    t = cb.Solver(m, config(inlet_rho=rho, inlet_u=u, inlet_v=v, inlet_p=p))
    t.set_option("persistent", 1)
    t.upload_state(U0)
    t.step(5)
    assert np.all(np.isfinite(t.download_U()))
