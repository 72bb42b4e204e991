"""The dense-block forward on the 5th-generation tensor cores (tcgen05.mma, accumulators in tensor
memory; cfd_mpnn_mlp_forward with engine = 1) against the mma.sync kernel (engine = 0) and the CPU
restatement with BF16 operands (oracle/mpnn_ref.py), for every block shape of the network: input
widths 9, 5, 192, 128 and 64 (gathered and plain segments), outputs 64 and 4, row counts that are
and are not multiples of the 128-row tile, and more tiles than thread blocks (each block then runs
several tiles, alternating the phases of its mbarrier)."""
import ctypes

import numpy as np
import pytest

import cfd_solver_withcuda_b200 as cb
from cfd_solver_withcuda_b200 import warmstart as ws

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-30))


@pytest.mark.parametrize("block,rows", [("enc_n", 1000), ("enc_e", 4096), ("edge0", 1000), ("edge0", 256),
                                        ("node0", 777), ("dec", 1000), ("edge0", 128 * 700 + 5),
                                        ("dec", 128 * 900)])
def test_tcgen05_forward_matches_mma_sync_and_restatement(block, rows):
    import torch
    from oracle import mpnn_ref as R
    rng = np.random.default_rng(hash(block) % 1000 + rows)
    P = R.init_params(9, 5, 4, 1, seed=3)
    K = P[block][0].shape[1]
    n_src = 300
    T = lambda a, dt=torch.float32: torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dt)
    if block == "edge0":
        h = rng.normal(size=(n_src, 64))
        e = rng.normal(size=(rows, 64))
        src, dst = rng.integers(0, n_src, rows), rng.integers(0, n_src, rows)
        th, te = T(h), T(e)
        segs = [ws._seg(th, T(src, torch.int32)), ws._seg(th, T(dst, torch.int32)), ws._seg(te)]
        x = np.concatenate([h[src], h[dst], e], axis=1)
    elif block == "node0":
        h, g = rng.normal(size=(rows, 64)), rng.normal(size=(rows, 64))
        segs = [ws._seg(T(h)), ws._seg(T(g))]
        x = np.concatenate([h, g], axis=1)
    else:
        x = rng.normal(size=(rows, K))
        segs = [ws._seg(T(x))]
    N2 = P[block][2].shape[0]
    outs = []
    for engine in (0, 1):
        net = ws.Net(layers=1, engine=engine)
        net.set_params(P)
        y = torch.full((rows, N2), np.nan, device="cuda")
        z1 = torch.full((rows, 64), np.nan, device="cuda")
        net._mlp(block, segs, rows, y, z1)
        torch.cuda.synchronize()
        outs.append((y.cpu().numpy(), z1.cpu().numpy()))
    st = ctypes.c_int(-1)
    cb._check(cb.lib().cfd_mpnn_status(ctypes.byref(st), 1))
    assert st.value == 0
    (y0, z0), (y1, z1_) = outs
    assert np.all(np.isfinite(y1)) and np.all(np.isfinite(z1_))
    yq, zq = R.mlp_forward(x, P[block], R.bf16)
    assert _rel(z1_, z0) < 1e-5 and _rel(y1, y0) < 1e-4
    assert _rel(z1_, zq) < 1e-5 and _rel(y1, yq) < 1e-4


def test_tcgen05_network_trains_like_mma_sync():
    """Whole network, forward through the tcgen05 blocks: the same prediction as the mma.sync
    blocks up to FP32 summation order, and a training run reduces the loss."""
    import torch
    P = ws.draw_parameters(4, 3)
    meshes = [ws.make_mesh(12, 6, t) for t, _, _ in P]
    g = ws.MeshGraph(meshes[0])
    feats = [g.features(m, p) for m, p in zip(meshes, P)]
    gb = ws.GraphBatch(g, 2, "cuda")
    xn = torch.from_numpy(np.concatenate([feats[0][0], feats[1][0]])).cuda()
    xe = torch.from_numpy(np.concatenate([feats[0][1], feats[1][1]])).cuda()
    preds = []
    for engine in (0, 1):
        net = ws.build_model(engine=engine)
        preds.append(net.forward(xn, xe, gb).cpu().numpy())
    assert _rel(preds[1], preds[0]) < 1e-3
    rng = np.random.default_rng(0)
    targets = [np.tanh(f[0][:, :4] + 0.1 * rng.normal(size=(g.N, 4))).astype(np.float32) for f in feats]
    net = ws.build_model(engine=1)
    losses = ws.train(net, g, [f[0] for f in feats], [f[1] for f in feats], targets, epochs=20, batch=2)
    assert losses[-1] < 0.5 * losses[0], losses


@pytest.mark.parametrize("K,N2,rows", [(9, 64, 1000), (5, 64, 4096), (192, 64, 1000), (192, 64, 128 * 300 + 7),
                                       (128, 64, 777), (64, 4, 1000), (64, 4, 128 * 200)])
def test_tcgen05_backward_matches_mma_sync_and_restatement(K, N2, rows):
    """The backward data path (dz1 = (dy W2) * silu'(z1), dx = dz1 W1) on tcgen05 (engine 1)
    against the mma.sync kernel (engine 0) and the CPU restatement with BF16 operands, for every
    block shape of the network, with and without dx."""
    import torch
    from oracle import mpnn_ref as R
    rng = np.random.default_rng(K * 1000 + N2 + rows)
    W1, W2 = rng.normal(size=(64, K)) / np.sqrt(K), rng.normal(size=(N2, 64)) / 8.0
    dy, z1 = rng.normal(size=(rows, N2)), rng.normal(size=(rows, 64))
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    tw1, tw2, tdy, tz1 = T(W1), T(W2), T(dy), T(z1)
    outs = []
    for engine in (0, 1):
        for with_dx in (True, False):
            dz1 = torch.full((rows, 64), np.nan, device="cuda")
            dx = torch.full((rows, K), np.nan, device="cuda") if with_dx else None
            a = cb.MlpBwd()
            a.rows, a.in_width, a.out = rows, K, N2
            a.dy, a.ld_dy, a.z1 = tdy.data_ptr(), N2, tz1.data_ptr()
            a.w1, a.w2, a.dz1 = tw1.data_ptr(), tw2.data_ptr(), dz1.data_ptr()
            a.dx, a.ld_dx = (dx.data_ptr(), K) if with_dx else (None, 0)
            a.engine = engine
            cb._check(cb.lib().cfd_mpnn_mlp_backward(ctypes.byref(a), None))
            torch.cuda.synchronize()
            outs.append((dz1.cpu().numpy(), dx.cpu().numpy() if with_dx else None))
    st = ctypes.c_int(-1)
    cb._check(cb.lib().cfd_mpnn_status(ctypes.byref(st), 1))
    assert st.value == 0
    dz_ref = (R.bf16(dy.astype(np.float32)) @ R.bf16(W2.astype(np.float32))) * R.dsilu(z1.astype(np.float32))
    dx_ref = R.bf16(dz_ref) @ R.bf16(W1.astype(np.float32))
    (dz0, dx0), (dz0b, _), (dz1_, dx1), (dz1b, _) = outs
    assert np.all(np.isfinite(dz1_)) and np.all(np.isfinite(dx1))
    assert np.array_equal(dz1_, dz1b) and np.array_equal(dz0, dz0b)
    assert _rel(dz1_, dz0) < 1e-5 and _rel(dx1, dx0) < 1e-4
    assert _rel(dz1_, dz_ref) < 1e-5 and _rel(dx1, dx_ref) < 1e-4
