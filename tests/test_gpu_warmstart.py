"""Warm-start surrogate: its library kernels (deterministic segment sums, fused Adam), the
gradients of the graph operations, the batch machinery it relies on (per-member boundary values,
shared residual normalisers) and a small end-to-end run."""
import numpy as np
import pytest

import cfd_solver_withcuda_b200 as cb
from cfd_solver_withcuda_b200 import warmstart as ws

pytestmark = pytest.mark.gpu


def _csr(rng, n_rows, n_items, max_per_row=5):
    counts = rng.integers(0, max_per_row + 1, n_rows)
    ptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    idx = rng.integers(0, n_items, ptr[-1]).astype(np.int32)
    return ptr, idx


def test_segment_sum_matches_direct_sums_and_is_deterministic():
    import torch
    rng = np.random.default_rng(1)
    x = rng.normal(size=(3000, 64)).astype(np.float32)
    ptr, idx = _csr(rng, 1000, 3000)
    want = np.zeros((1000, 64), np.float64)
    for r in range(1000):
        for j in range(ptr[r], ptr[r + 1]):
            want[r] += x[idx[j]]
    t = lambda a: torch.from_numpy(a).cuda()
    a = ws.segment_sum(t(x), t(ptr), t(idx), 1000).cpu().numpy()
    b = ws.segment_sum(t(x), t(ptr), t(idx), 1000).cpu().numpy()
    np.testing.assert_allclose(a, want, rtol=1e-5, atol=1e-5)
    assert np.array_equal(a.view(np.int32), b.view(np.int32))


def test_adam_step_matches_formula():
    import torch
    rng = np.random.default_rng(2)
    p0 = rng.normal(size=500).astype(np.float32)
    grads = [rng.normal(size=500).astype(np.float32) for _ in range(3)]
    p = torch.nn.Parameter(torch.from_numpy(p0.copy()).cuda())
    opt = ws.Adam([p], lr=1e-2)
    m = np.zeros(500)
    v = np.zeros(500)
    q = p0.astype(np.float64)
    for t, g in enumerate(grads, start=1):
        p.grad = torch.from_numpy(g).cuda()
        opt.step()
        m = 0.9 * m + 0.1 * g
        v = 0.999 * v + 0.001 * g.astype(np.float64) ** 2
        q -= 1e-2 * (m / (1 - 0.9 ** t)) / (np.sqrt(v / (1 - 0.999 ** t)) + 1e-8)
    np.testing.assert_allclose(p.detach().cpu().numpy(), q, rtol=1e-5, atol=1e-6)


def test_graph_operations_gradients_match_torch_reference():
    """Gather and Aggregate (custom backward through the segment sums) against torch's own
    index_select / index_add on the same data."""
    import torch
    m = ws.make_mesh(12, 6, 0.1)
    g = ws.MeshGraph(m)
    gb = ws.GraphBatch(g, 2, "cuda")
    Gather, Aggregate = ws._functions()
    rng = np.random.default_rng(3)
    h0 = torch.from_numpy(rng.normal(size=(2 * g.N, 8)).astype(np.float32)).cuda()
    w = torch.from_numpy(rng.normal(size=(2 * g.E, 8)).astype(np.float32)).cuda()

    def ours(h):
        hs = Gather.apply(h, gb.src, gb.src_ptr, gb.src_order)
        hd = Gather.apply(h, gb.dst, gb.dst_ptr, gb.ident)
        agg = Aggregate.apply(hs * w + hd, gb.dst_ptr, gb.ident, gb.dst)
        return (agg ** 2).sum()

    def ref(h):
        hs = h.index_select(0, gb.src.long())
        hd = h.index_select(0, gb.dst.long())
        agg = torch.zeros_like(h).index_add_(0, gb.dst.long(), hs * w + hd)
        return (agg ** 2).sum()

    a = h0.clone().requires_grad_(True)
    b = h0.clone().requires_grad_(True)
    la, lb = ours(a), ref(b)
    la.backward()
    lb.backward()
    np.testing.assert_allclose(float(la.detach()), float(lb.detach()), rtol=1e-5)
    np.testing.assert_allclose(a.grad.cpu().numpy(), b.grad.cpu().numpy(), rtol=1e-4, atol=1e-4)


def test_restart_from_converged_states_meets_the_shared_tolerance_at_once():
    """Members solved to a tolerance, then restarted from their own converged states with the
    freestream normalisers: every member meets the tolerance at the first check."""
    P = ws.draw_parameters(3, 5)
    meshes = [ws.make_mesh(16, 8, t) for t, _, _ in P]
    fs = [ws.freestream_state(m, M) for m, (_, M, _) in zip(meshes, P)]
    r0 = ws.first_residuals(meshes, P, fs)
    res, U, _ = ws.solve(meshes, P, fs, tol=1e-2, max_steps=20000, check_every=100, r0=r0)
    assert np.all(res["steps_to_tol"] > 0), res
    res2, _, _ = ws.solve(meshes, P, U, tol=1e-2, max_steps=2000, check_every=100, r0=r0)
    assert np.all((res2["steps_to_tol"] > 0) & (res2["steps_to_tol"] <= 101)), res2


def test_per_member_boundary_values_equal_single_solves():
    """A batch with per-member total-(p, T) inflow and exit pressure gives each member the same
    bits as a single solve configured with that member's values."""
    P = ws.draw_parameters(3, 9)
    meshes = [ws.make_mesh(16, 8, t) for t, _, _ in P]
    fs = [ws.freestream_state(m, M) for m, (_, M, _) in zip(meshes, P)]
    res, U, _ = ws.solve(meshes, P, fs, tol=0.0, max_steps=40, check_every=40)
    for m, U0, Ub, (_, M, r) in zip(meshes, fs, U, P):
        p0, T0, pe = ws.boundary_values(M, r)
        s = cb.Solver(m, ws.solver_config(inlet_p0=p0, inlet_t0=T0, exit_p=pe))
        s.upload_state(U0)
        s.step(40)
        assert np.array_equal(s.download_U().view(np.int64), Ub.view(np.int64))


def test_warm_start_experiment_small():
    out = ws.run_experiment(nx=16, ny=8, n_train=8, n_test=3, tol=1e-2, max_steps=20000, check_every=100, epochs=5,
                            batch=4)
    assert out["parameters"] > 150000
    assert out["train_converged"] == 8 and out["freestream_converged"] == 3
    assert 0.0 <= out["fallback_rate"] <= 1.0
    assert np.isfinite(out["loss_last"]) and np.isfinite(out["prediction_rel_l2_median"])
