"""Warm-start surrogate: its library kernels (dense blocks on the tensor cores, deterministic
segment sums, fused Adam) checked against the CPU FP64 restatement oracle/mpnn_ref.py (single
blocks and whole-network gradients), the batch machinery it relies on (per-member boundary values,
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
    import ctypes
    import torch
    rng = np.random.default_rng(2)
    p0 = rng.normal(size=500).astype(np.float32)
    grads = [rng.normal(size=500).astype(np.float32) for _ in range(3)]
    p = torch.from_numpy(p0.copy()).cuda()
    mt, vt = torch.zeros_like(p), torch.zeros_like(p)
    m = np.zeros(500)
    v = np.zeros(500)
    q = p0.astype(np.float64)
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    for t, g in enumerate(grads, start=1):
        gt = torch.from_numpy(g).cuda()
        cb._check(cb.lib().cfd_mpnn_adam(vp(p), vp(gt), vp(mt), vp(vt), 500, 1e-2, 0.9, 0.999, 1e-8, t, None))
        m = 0.9 * m + 0.1 * g
        v = 0.999 * v + 0.001 * g.astype(np.float64) ** 2
        q -= 1e-2 * (m / (1 - 0.9 ** t)) / (np.sqrt(v / (1 - 0.999 ** t)) + 1e-8)
    np.testing.assert_allclose(p.cpu().numpy(), q, rtol=1e-5, atol=1e-6)


def _graph_batch(nx, ny, B):
    g = ws.MeshGraph(ws.make_mesh(nx, ny, 0.08))
    gb = ws.GraphBatch(g, B, "cuda")
    host = {k: getattr(gb, k).cpu().numpy().astype(np.int64) for k in ("src", "dst", "dst_ptr")}
    return g, gb, host


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-30))


def test_dense_block_kernels_match_cpu_restatement():
    """One dense block with gathered input segments: forward (y, z1), backward data (dz1, dx) and
    weight gradients (dW1, db1, dW2, db2) against the CPU FP64 restatement with the kernels' BF16
    operand rounding (tight: only the FP32 accumulation differs) and without it (loose)."""
    import torch
    from oracle import mpnn_ref as R
    rng = np.random.default_rng(11)
    rows, n_src = 1000, 300
    h = rng.normal(size=(n_src, 64))
    e = rng.normal(size=(rows, 64))
    src = rng.integers(0, n_src, rows)
    dst = rng.integers(0, n_src, rows)
    net = ws.Net(layers=1)
    P = R.init_params(9, 5, 4, 1, seed=5)
    net.set_params(P)
    p = P["edge0"]
    x = np.concatenate([h[src], h[dst], e], axis=1)
    T = lambda a, dt=torch.float32: torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dt)
    th, te, ts, td = T(h), T(e), T(src, torch.int32), T(dst, torch.int32)
    y = torch.empty((rows, 64), device="cuda")
    z1 = torch.empty((rows, 64), device="cuda")
    net._mlp("edge0", [ws._seg(th, ts), ws._seg(th, td), ws._seg(te)], rows, y, z1, resid=te)
    q = R.bf16
    yq, zq = R.mlp_forward(x, p, q)
    y64, z64 = R.mlp_forward(x, p, lambda a: a)
    assert _rel(z1.cpu().numpy(), zq) < 1e-5 and _rel(y.cpu().numpy(), yq + e) < 1e-5
    assert _rel(y.cpu().numpy(), y64 + e) < 1e-2
    dy = rng.normal(size=(rows, 64))
    net._bufs = {"dz": torch.empty((rows, 64), device="cuda")}
    dx = torch.empty((rows, 192), device="cuda")
    net._block_grads("edge0", T(dy), z1, rows, [ws._seg(th, ts), ws._seg(th, td), ws._seg(te)], dx=dx)
    dxq, gq = R.mlp_backward(x, z1.cpu().numpy().astype(np.float64), dy, p, q)
    assert _rel(dx.cpu().numpy(), dxq) < 1e-4
    got = [t.cpu().numpy() for t in net.g["edge0"]]
    for a, b in zip(got, gq):
        assert _rel(a, b) < 1e-4
    _, g64 = R.mlp_backward(x, z64, dy, p, lambda a: a)
    for a, b in zip(got, g64):
        assert _rel(a, b) < 3e-2


def test_network_gradients_match_cpu_fp64_restatement():
    """The whole network (2 message-passing layers on two stacked mesh graphs): loss and every
    parameter gradient of the library's kernels against the CPU restatement, with BF16 operand
    rounding emulated (tight) and in exact FP64 (loose: BF16 operands)."""
    import torch
    from oracle import mpnn_ref as R
    layers = 2
    g, gb, hg = _graph_batch(12, 6, 2)
    rng = np.random.default_rng(4)
    xn = rng.normal(size=(2 * g.N, 9))
    xe = rng.normal(size=(2 * g.E, 5))
    target = rng.normal(size=(2 * g.N, 4))
    P = R.init_params(9, 5, 4, layers, seed=9)
    net = ws.Net(layers=layers)
    net.set_params(P)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    pred = net.forward(T(xn), T(xe), gb)
    loss, dpred = net.loss_grad(T(target))
    net.backward(dpred)
    G = net.get_grads()
    Lq, predq, Gq = R.loss_and_grad(P, xn, xe, hg["src"], hg["dst"], hg["dst_ptr"], target, layers, use_bf16=True)
    L64, pred64, G64 = R.loss_and_grad(P, xn, xe, hg["src"], hg["dst"], hg["dst_ptr"], target, layers)
    # BF16-emulated restatement: the FP32 accumulation order of the kernels can flip the BF16
    # rounding of an activation, so the agreement is ~1e-4 relative rather than to the last bit.
    assert _rel(pred.cpu().numpy(), predq) < 1e-3
    assert abs(float(loss) - Lq) <= 1e-3 * Lq
    assert _rel(pred.cpu().numpy(), pred64) < 2e-2
    for name in net.names:
        for part in range(4):
            a, bq, b64 = G[name][part], Gq[name][part], G64[name][part]
            assert _rel(a, bq) < 5e-3, (name, part, _rel(a, bq))
            assert _rel(a, b64) < 5e-2, (name, part, _rel(a, b64))
    # Repeatable to the bit.
    net.forward(T(xn), T(xe), gb)
    net.loss_grad(T(target))
    net.backward(net._bufs["dpred"])
    G2 = net.get_grads()
    for name in net.names:
        for a, b in zip(G[name], G2[name]):
            assert np.array_equal(a, b)


def test_training_with_library_kernels_reduces_the_loss():
    P = ws.draw_parameters(6, 3)
    meshes = [ws.make_mesh(12, 6, t) for t, _, _ in P]
    g = ws.MeshGraph(meshes[0])
    feats = [g.features(m, p) for m, p in zip(meshes, P)]
    rng = np.random.default_rng(0)
    targets = [np.tanh(f[0][:, :4] + 0.1 * rng.normal(size=(g.N, 4))).astype(np.float32) for f in feats]
    net = ws.build_model()
    losses = ws.train(net, g, [f[0] for f in feats], [f[1] for f in feats], targets, epochs=30, batch=3)
    assert losses[-1] < 0.3 * losses[0], losses


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
    out = ws.run_experiment(nx=16, ny=8, n_train=8, n_test=3, tol=1e-3, max_steps=20000, check_every=100, epochs=5,
                            batch=4, switch_tol=1e-2, n_plain=2)
    assert out["parameters"] > 150000
    assert out["train_converged"] == 8 and out["plain_converged"] == 2 and out["chosen_converged"] == 3
    assert 0.0 <= out["fallback_rate"] <= 1.0
    assert np.isfinite(out["loss_last"]) and np.isfinite(out["prediction_rel_l2_median"])
    assert out["speedup_chosen_vs_plain"] > 0.0
    # Both paths reach the same absolute residual target; their steady states agree closely.
    assert out["final_state_rel_l2_vs_plain_max"] < 1e-2


def test_divergence_guard_stops_a_growing_member():
    """A member whose residual ratio exceeds the batch's divergence_ratio stops with steps_to_tol
    -2: a member started from a state far from its steady state, guarded with a ratio below its
    early residual growth."""
    P = ws.draw_parameters(2, 13)
    meshes = [ws.make_mesh(16, 8, t) for t, _, _ in P]
    fs = [ws.freestream_state(m, M) for m, (_, M, _) in zip(meshes, P)]
    r0 = ws.first_residuals(meshes, P, fs)
    # Normalisers a thousand times smaller than the freestream's first residual: every ratio is
    # far above the guard at the first check.
    res, _, _ = ws.solve(meshes, P, fs, tol=1e-12, max_steps=400, check_every=100, r0=r0 * 1e-3, diverge=10.0)
    assert np.all(res["steps_to_tol"] == -2), res
