"""Known answers of the gradient-MUSCL face form, independent of the C restatement.

On a uniform Cartesian mesh the Green-Gauss gradient of a linear field is exact, so the upwind
difference D- = 2 grad q . d - D+ equals D+, every limiter gives phi(1) = 1, and the two
reconstructed face states are both the field's value at the face midpoint.  The Roe, HLLC and AUSM
fluxes of two equal states are the physical Euler flux, so every interior cell's residual must be
sum_f F(q(x_f)) . n_f dl_f, computed here from the primitives with numpy.  (Green-Gauss with
centre averages is exact for linear fields only where the midpoint of two centres is the face
centre, so a distorted mesh would not give a known answer.)"""
import numpy as np
import pytest

import cfd_solver_withcuda_b200 as cb

pytestmark = pytest.mark.gpu

GAMMA = 1.4
NX, NY = 24, 16


def linear_primitives(xy):
    x, y = xy[:, 0], xy[:, 1]
    rho = 1.0 + 0.10 * x + 0.05 * y
    u = 0.30 + 0.10 * x - 0.05 * y
    v = -0.20 + 0.04 * x + 0.10 * y
    p = 1.0 + 0.20 * x - 0.10 * y
    return rho, u, v, p


def euler_flux(rho, u, v, p, nx, ny):
    vn = u * nx + v * ny
    E = p / (GAMMA - 1.0) + 0.5 * rho * (u * u + v * v)
    return np.stack([rho * vn, rho * u * vn + p * nx, rho * v * vn + p * ny, (E + p) * vn], axis=-1)


def exact_residual(m, inner):
    """Per cell: sum_f F(q(x_f)) . n_f dl_f at the face midpoints, and sum_f |F . n_f dl_f| (the
    size of the face fluxes the residual is the small difference of)."""
    NP = m.n_physical
    want = np.zeros((NP, 4))
    scale = np.zeros(NP)
    for c in np.nonzero(inner)[0]:
        for f in range(m.n_faces[c]):
            n = m.neighbours[c, f]
            mid = 0.5 * (m.centers[c, :2] + m.centers[n, :2])
            q = linear_primitives(mid[None, :])
            F = euler_flux(*(a[0] for a in q), m.face_normals[c, 2 * f], m.face_normals[c, 2 * f + 1])
            F = F * m.face_lengths[c, f]
            want[c] += F
            scale[c] += np.abs(F).sum()
    return want, scale


def interior_cells(m):
    """Cells whose own faces, and whose neighbours' gradients, involve no ghost cell."""
    NP = m.n_physical
    inner = np.zeros(NP, bool)
    for c in range(NP):
        nb = m.neighbours[c, :m.n_faces[c]]
        if np.all(nb < NP) and all(np.all(m.neighbours[n, :m.n_faces[n]] < NP) for n in nb):
            inner[c] = True
    return inner


@pytest.mark.parametrize("limiter", [cb.LIM_MINMOD, cb.LIM_VANLEER, cb.LIM_SUPERBEE, cb.LIM_VANALBADA])
@pytest.mark.parametrize("dissipation", [cb.DISS_ROE, cb.DISS_HLLC, cb.DISS_AUSM])
@pytest.mark.parametrize("reorder", [0, 4])
def test_linear_field_gives_the_exact_face_flux(dissipation, limiter, reorder):
    m = cb.Mesh.box(NX, NY, 0.0, 1.5, 0.0, 1.0)
    NP = m.n_physical
    rho, u, v, p = linear_primitives(m.centers[:, :2])
    U0 = cb.conserved_from_primitive(rho, u, v, p)
    s = cb.Solver(m, cb.default_config(device=0, dissipation_type=dissipation, is_second_order=1,
                                       muscl=cb.MUSCL_GRADIENT, limiter=limiter, time_accurate=1,
                                       local_time_stepping=1, integrator=cb.INT_SSPRK3, cfl=0.5,
                                       reorder=reorder))
    s.upload_state(U0)
    s.Evaluate_Cell_Net_Flux()
    got = s.download()["net_flux"]

    inner = interior_cells(m)
    assert inner.sum() == (NX - 4) * (NY - 4)
    want, scale = exact_residual(m, inner)
    err = np.abs(got[inner] - want[inner]).max(axis=1) / scale[inner]
    assert err.max() < 1e-12, err.max()


def test_fp32_flux_form_within_float_rounding():
    m = cb.Mesh.box(NX, NY, 0.0, 1.5, 0.0, 1.0)
    rho, u, v, p = linear_primitives(m.centers[:, :2])
    U0 = cb.conserved_from_primitive(rho, u, v, p)
    out = []
    for prec in (cb.PREC_FP64, cb.PREC_FP32_FLUX):
        s = cb.Solver(m, cb.default_config(device=0, dissipation_type=cb.DISS_ROE, is_second_order=1,
                                           muscl=cb.MUSCL_GRADIENT, limiter=cb.LIM_VANLEER, time_accurate=1,
                                           local_time_stepping=1, integrator=cb.INT_SSPRK3, cfl=0.5,
                                           precision=prec))
        s.upload_state(U0)
        s.Evaluate_Cell_Net_Flux()
        out.append(s.download()["net_flux"])
    inner = interior_cells(m)
    want, scale = exact_residual(m, inner)
    err = np.abs(out[1][inner] - want[inner]).max(axis=1) / scale[inner]
    assert err.max() < 1e-6, err.max()
