"""Test infrastructure only: CPU FP64 restatement of the warm-start surrogate (the message-passing
network of cfd_solver_withcuda_b200/warmstart.py), forward pass and analytic backward pass.

It is the checker of the network's CUDA kernels (csrc/mpnn_tc.cu, csrc/mpnn.cu): with bf16=True
the operands are rounded to BF16 at the points where the kernels round them (inputs of every
matrix product), everything else is FP64, so the kernels' FP32 accumulation is the only other
difference; with bf16=False it is the exact FP64 network, whose gradients the tests also check
by central finite differences.

Network (no reference counterpart): blocks are two-layer perceptrons
    mlp(x) = W2 silu(W1 x + b1) + b2,  silu(z) = z / (1 + exp(-z)),  hidden width 64;
    h = enc_n(x_node), e = enc_e(x_edge);
    layer l: e <- e + edge_l([h[src], h[dst], e]);  agg[n] = sum of e over edges with dst = n
             (edges sorted by destination); h <- h + node_l([h, agg]);
    prediction = dec(h); loss = mean((prediction - target)^2).
Parameters: dict name -> (W1 [64][K], b1 [64], W2 [N][64], b2 [N]) for the names enc_n, enc_e,
edge0..edge{L-1}, node0..node{L-1}, dec.
"""
import numpy as np

HIDDEN = 64


def bf16(x):
    """Round float64 values to the nearest BF16 (ties to even) through float32, as the kernels do
    (__float2bfloat16_rn of the float32 operand)."""
    f = np.ascontiguousarray(np.asarray(x, np.float64).astype(np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def block_names(layers):
    return ["enc_n", "enc_e"] + ["edge%d" % l for l in range(layers)] + ["node%d" % l for l in range(layers)] + ["dec"]


def init_params(node_in, edge_in, out, layers, seed, width=HIDDEN):
    """Uniform(-1/sqrt(K), 1/sqrt(K)) weights and biases per linear layer (K = its input width)."""
    rng = np.random.default_rng(seed)
    dims = {"enc_n": (node_in, width), "enc_e": (edge_in, width), "dec": (width, out)}
    for l in range(layers):
        dims["edge%d" % l] = (3 * width, width)
        dims["node%d" % l] = (2 * width, width)
    P = {}
    for name in block_names(layers):
        K, N = dims[name]
        a, c = 1.0 / np.sqrt(K), 1.0 / np.sqrt(width)
        P[name] = (rng.uniform(-a, a, (width, K)), rng.uniform(-a, a, width),
                   rng.uniform(-c, c, (N, width)), rng.uniform(-c, c, N))
    return P


def mlp_forward(x, p, q):
    """(y, z1) of one block; q rounds matrix-product operands (identity or bf16)."""
    W1, b1, W2, b2 = p
    z1 = q(x) @ q(W1).T + b1
    y = q(silu(z1)) @ q(W2).T + b2
    return y, z1


def mlp_backward(x, z1, dy, p, q):
    """(dx, (dW1, db1, dW2, db2)) of one block, operands rounded as the kernels round them."""
    W1, b1, W2, b2 = p
    s = silu(z1)
    dW2 = q(dy).T @ q(s)
    db2 = dy.sum(axis=0)
    dz1 = (q(dy) @ q(W2)) * dsilu(z1)
    dW1 = q(dz1).T @ q(x)
    db1 = dz1.sum(axis=0)
    dx = q(dz1) @ q(W1)
    return dx, (dW1, db1, dW2, db2)


def segment_sum(x, ptr, n_rows):
    """Rows of x summed over the consecutive CSR ranges [ptr[r], ptr[r+1])."""
    out = np.zeros((n_rows, x.shape[1]))
    for r in range(n_rows):
        out[r] = x[ptr[r]:ptr[r + 1]].sum(axis=0)
    return out


def forward(P, xn, xe, src, dst, dst_ptr, layers, use_bf16=False):
    """Prediction and the activations the backward pass needs."""
    q = bf16 if use_bf16 else (lambda a: a)
    N = xn.shape[0]
    h, zn = mlp_forward(xn, P["enc_n"], q)
    e, ze = mlp_forward(xe, P["enc_e"], q)
    acts = {"enc_n": (xn, zn), "enc_e": (xe, ze)}
    for l in range(layers):
        xin = np.concatenate([h[src], h[dst], e], axis=1)
        y, z = mlp_forward(xin, P["edge%d" % l], q)
        acts["edge%d" % l] = (xin, z)
        e = e + y
        agg = segment_sum(e, dst_ptr, N)
        xin = np.concatenate([h, agg], axis=1)
        y, z = mlp_forward(xin, P["node%d" % l], q)
        acts["node%d" % l] = (xin, z)
        h = h + y
    pred, z = mlp_forward(h, P["dec"], q)
    acts["dec"] = (h, z)
    return pred, acts


def loss_and_grad(P, xn, xe, src, dst, dst_ptr, target, layers, use_bf16=False):
    """Mean-squared-error loss and the gradient of every parameter."""
    q = bf16 if use_bf16 else (lambda a: a)
    N, E, W = xn.shape[0], xe.shape[0], HIDDEN
    pred, acts = forward(P, xn, xe, src, dst, dst_ptr, layers, use_bf16)
    d = pred - target
    loss = float((d * d).mean())
    dpred = 2.0 * d / d.size
    G = {}
    x, z = acts["dec"]
    dh, G["dec"] = mlp_backward(x, z, dpred, P["dec"], q)
    de = np.zeros((E, W))
    for l in reversed(range(layers)):
        x, z = acts["node%d" % l]
        dx, G["node%d" % l] = mlp_backward(x, z, dh, P["node%d" % l], q)
        dh = dh + dx[:, :W]
        de = de + dx[:, W:2 * W][dst]
        x, z = acts["edge%d" % l]
        dx, G["edge%d" % l] = mlp_backward(x, z, de, P["edge%d" % l], q)
        dsrc, ddst = dx[:, :W], dx[:, W:2 * W]
        np.add.at(dh, src, dsrc)
        np.add.at(dh, dst, ddst)
        de = de + dx[:, 2 * W:]
    x, z = acts["enc_e"]
    _, G["enc_e"] = mlp_backward(x, z, de, P["enc_e"], q)
    x, z = acts["enc_n"]
    _, G["enc_n"] = mlp_backward(x, z, dh, P["enc_n"], q)
    return loss, pred, G
