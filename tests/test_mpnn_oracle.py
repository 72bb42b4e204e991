"""The CPU FP64 restatement of the warm-start network (oracle/mpnn_ref.py), which checks the
network's CUDA kernels, checked itself: its analytic gradients against central finite
differences of its own loss, for every parameter block, and its BF16 rounding against the format's
definition."""
import numpy as np

from oracle import mpnn_ref as R


def _graph(rng, n_nodes=9, n_edges=30):
    dst = np.sort(rng.integers(0, n_nodes, n_edges))
    src = rng.integers(0, n_nodes, n_edges)
    ptr = np.zeros(n_nodes + 1, np.int64)
    np.add.at(ptr, dst + 1, 1)
    return src, dst, np.cumsum(ptr)


def test_analytic_gradients_match_finite_differences():
    rng = np.random.default_rng(7)
    layers = 2
    src, dst, ptr = _graph(rng)
    xn = rng.normal(size=(9, 9))
    xe = rng.normal(size=(30, 5))
    target = rng.normal(size=(9, 4))
    P = R.init_params(9, 5, 4, layers, seed=3)
    loss, _, G = R.loss_and_grad(P, xn, xe, src, dst, ptr, target, layers)
    eps = 1e-6
    for name in R.block_names(layers):
        for part in range(4):
            arr = P[name][part]
            for _ in range(3):
                idx = tuple(rng.integers(0, s) for s in arr.shape)
                old = arr[idx]
                arr[idx] = old + eps
                lp = R.loss_and_grad(P, xn, xe, src, dst, ptr, target, layers)[0]
                arr[idx] = old - eps
                lm = R.loss_and_grad(P, xn, xe, src, dst, ptr, target, layers)[0]
                arr[idx] = old
                fd = (lp - lm) / (2 * eps)
                an = G[name][part][idx]
                assert abs(fd - an) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (name, part, idx, fd, an)


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -7 + 2 ** -9, -3.14159265, 1e-30, 65504.0])
    r = R.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == 1.0 + 2 ** -7  # a quarter of a unit above 1 + 2^-7 rounds down
    u = r.astype(np.float32).view(np.uint32)
    assert np.all((u & 0xFFFF) == 0)
    assert np.all(np.abs(r - x) <= np.abs(x) * 2 ** -8)
