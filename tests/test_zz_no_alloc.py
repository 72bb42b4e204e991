"""cfd_evaluate_net_flux_noalloc: the residual evaluation for callers that cannot let the library
allocate device memory (their own pool allocator owns the GPU's memory, or their loop cannot take
cudaMalloc's device synchronisation).  The test owns every device array (allocated here with
torch), calls the entry point through the C ABI twice in a row on two different states, and
checks each result bit for bit against the existing entry point, cfd_evaluate_net_flux, of a
context on the same mesh and state, and that calls after the first take no device memory (free
device memory unchanged across a call, also on another stream).  This file is collected last on
purpose."""
import ctypes

import numpy as np
import pytest

import cfd_solver_withcuda_b200 as cb
from cases import CASES, initial_state, make_mesh, solver_config
from conftest import assert_bits_equal

pytestmark = pytest.mark.gpu


def limiter_stencil(m):
    """N2, d1, d2 of the reference's Second_Order_Limiter (src/Limiters.cpp:136-191), face-major."""
    NP = m.n_physical
    n2 = np.zeros((4, NP), np.int32)
    d1 = np.ones((4, NP))
    d2 = np.ones((4, NP))
    for c in range(NP):
        for f in range(m.n_faces[c]):
            N = m.neighbours[c, f]
            a = m.center_distances[c, f]
            if m.n_faces[c] != 4:
                a = 1.0 if a <= 0.0 else a
                n2[f, c], d1[f, c], d2[f, c] = N, a, a
            elif f < 2:
                ghost = N >= NP
                n2[f, c] = N if ghost else m.neighbours[N, f]
                d1[f, c] = a
                d2[f, c] = a if ghost else m.center_distances[N, f]
            else:
                n2[f, c] = m.neighbours[c, f - 2]
                d1[f, c] = a
                d2[f, c] = m.center_distances[c, f - 2]
    return n2, d1, d2


@pytest.mark.parametrize("over", [{}, dict(dissipation_type=2, movers_entropy_fix=1), dict(dissipation_type=4),
                                  dict(dissipation_type=5), dict(dissipation_type=2, is_second_order=0,
                                                                 movers_single_alpha=1)])
def test_noalloc_matches_context_on_two_calls(over):
    import torch
    case = CASES["cyl_roe2_lts"]
    m = make_mesh(case)
    NP, NT = m.n_physical, m.n_total
    cfg = solver_config(case, reorder=0, **over)
    s = cb.Solver(m, cfg)
    s.upload_state(initial_state(case, m))

    dev = torch.device("cuda", 0)

    def on_dev(a, dtype):
        return torch.from_numpy(np.ascontiguousarray(a)).to(device=dev, dtype=dtype)

    nbr = np.zeros((4, NP), np.int32)
    nx = np.zeros((4, NP))
    ny = np.zeros((4, NP))
    dl = np.zeros((4, NP))
    degen = np.zeros(NP, np.uint8)
    for f in range(4):
        has = m.n_faces > f
        nbr[f, has] = m.neighbours[has, f]
        nx[f, has] = m.face_normals[has, 2 * f]
        ny[f, has] = m.face_normals[has, 2 * f + 1]
        dl[f, has] = m.face_lengths[has, f]
        degen |= (has & (np.sqrt(nx[f] * nx[f] + ny[f] * ny[f]) < 1e-12)).astype(np.uint8) << f
    n2, d1, d2 = limiter_stencil(m)
    keep = {"n_faces": on_dev(m.n_faces.astype(np.int32), torch.int32), "neighbours": on_dev(nbr, torch.int32),
            "nx": on_dev(nx, torch.float64), "ny": on_dev(ny, torch.float64), "dl": on_dev(dl, torch.float64),
            "area": on_dev(m.area, torch.float64), "inv_area": on_dev(m.inv_area, torch.float64),
            "second_neighbours": on_dev(n2, torch.int32), "d1": on_dev(d1, torch.float64),
            "d2": on_dev(d2, torch.float64), "degenerate": on_dev(degen, torch.uint8),
            "net_flux": torch.zeros((4, NP), dtype=torch.float64, device=dev),
            "dt": torch.zeros(NP, dtype=torch.float64, device=dev),
            "min_dt": torch.zeros(1, dtype=torch.float64, device=dev)}

    for call in range(2):
        if call == 1:
            s.step(3)  # a different state for the second call
        s.Apply_Boundary_Conditions()
        st = s.download()
        s.Evaluate_Cell_Net_Flux()
        want = s.download()
        want_min_dt = s.get_Min_dt()
        keep["prim"] = on_dev(st["prim"][:, [0, 1, 2, 4, 5]].T, torch.float64)
        keep["U"] = on_dev(st["U"].T, torch.float64)
        keep["net_flux"].fill_(np.nan)
        keep["dt"].fill_(np.nan)
        keep["min_dt"].fill_(np.nan)
        a = cb.FluxArrays()
        a.n_physical, a.n_total = NP, NT
        for name, t in keep.items():
            setattr(a, name, t.data_ptr())
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info(dev)[0]
        rc = cb.lib().cfd_evaluate_net_flux_noalloc(ctypes.byref(a), ctypes.byref(cfg), None)
        assert rc == cb.CFD_OK, cb.lib().cfd_last_error()
        torch.cuda.synchronize()
        if call == 1:
            # The first call may load the library's device code into this context (which places
            # the static scratch array); from then on a call takes no device memory.
            assert torch.cuda.mem_get_info(dev)[0] == free_before, "the second call changed free device memory"
        assert_bits_equal(keep["net_flux"].cpu().numpy().T, want["net_flux"], "net flux, call %d" % call)
        assert_bits_equal(keep["dt"].cpu().numpy(), want["dt"], "del_t, call %d" % call)
        assert_bits_equal(keep["min_dt"].cpu().numpy(), np.array([want_min_dt]), "Min_dt, call %d" % call)

    # A further call on a stream of its own: same results as the second call, no device memory.
    side = torch.cuda.Stream(device=dev)
    want_flux = keep["net_flux"].clone()
    keep["net_flux"].fill_(np.nan)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(dev)[0]
    rc = cb.lib().cfd_evaluate_net_flux_noalloc(ctypes.byref(a), ctypes.byref(cfg), ctypes.c_void_p(side.cuda_stream))
    assert rc == cb.CFD_OK, cb.lib().cfd_last_error()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(dev)[0] == free_before, "a call on another stream changed free device memory"
    assert_bits_equal(keep["net_flux"].cpu().numpy(), want_flux.cpu().numpy(), "net flux on a second stream")


def test_noalloc_rejects_sizes_beyond_its_scratch():
    a = cb.FluxArrays()
    a.n_physical, a.n_total = 8388608 + 1, 8388608 + 10
    rc = cb.lib().cfd_evaluate_net_flux_noalloc(ctypes.byref(a), ctypes.byref(cb.default_config()), None)
    assert rc == 1
    assert b"8388608" in cb.lib().cfd_last_error()
