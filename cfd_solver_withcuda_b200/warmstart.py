"""Learned warm start for families of steady solves (no reference counterpart).

The problem family: a 3 x 1 channel with a circular-arc bump of chord 1 and thickness t on the
lower wall, a structured quad mesh morphed to each t (same connectivity for every member), a
total-pressure / total-temperature inflow given by the inlet Mach number M of a (rho = 1,
p = 1/1.4) stream, and a static back pressure p_b = ratio * p0 at the exit.  Members are solved
to steady state by the batched FP64 solver (cfd_batch_*).  A message-passing network on the mesh's
cell graph (cells as nodes, faces as directed edges) maps (geometry, t, M, ratio) to the steady
(rho, u, v, p); its prediction is the start state of a new solve.

The network: node and edge encoders, L message-passing layers (edge update from the two end
cells and the edge, aggregation of the incoming messages of each cell in a fixed order, node
update), a decoder; width 64, SiLU, residual updates.  Forward, backward and optimiser are the
library's own kernels: the dense blocks on the tensor cores with BF16 operands and FP32
accumulation (cfd_mpnn_mlp_forward / _backward / cfd_mpnn_weight_grad), the graph operations as
deterministic segment sums and gathers, the loss gradient and a fused Adam step.  torch only
allocates the device buffers.
"""
import ctypes
import time

import numpy as np

import cfd_solver_withcuda_b200 as cb

GAMMA = 1.4
R_GAS = 287.0
LENGTH, HEIGHT = 3.0, 1.0


# ---------------------------------------------------------------------------------------------
# Problem family and solves
# ---------------------------------------------------------------------------------------------
def draw_parameters(n, seed, t_range=(0.04, 0.12), mach_range=(0.5, 0.8), ratio_range=(0.85, 1.0)):
    """n draws of (thickness, inlet Mach, back-pressure ratio p_b / p0), uniform, seeded."""
    rng = np.random.default_rng(seed)
    return np.stack([rng.uniform(*t_range, n), rng.uniform(*mach_range, n), rng.uniform(*ratio_range, n)], axis=1)


def make_mesh(nx, ny, thickness):
    """Structured quad bump channel morphed to `thickness` (same cell numbering for every t)."""
    return cb.Mesh.bump(nx, ny, LENGTH, HEIGHT, float(thickness), 0, 0.0, 0, False)


def boundary_values(mach, ratio):
    """(p0, T0, p_exit) of the member: total state of a (rho = 1, p = 1/1.4) stream at `mach`."""
    rho, p = 1.0, 1.0 / GAMMA
    T = p / (rho * R_GAS)
    f = 1.0 + 0.5 * (GAMMA - 1.0) * mach * mach
    p0 = p * f ** (GAMMA / (GAMMA - 1.0))
    return p0, T * f, ratio * p0


def freestream_state(mesh, mach):
    """Uniform (rho = 1, u = M a, v = 0, p = 1/1.4) on every row, ghosts included."""
    rho, p = 1.0, 1.0 / GAMMA
    u = mach * np.sqrt(GAMMA * p / rho)
    NT = mesh.n_total
    return cb.conserved_from_primitive(np.full(NT, rho), np.full(NT, u), np.zeros(NT), np.full(NT, p))


def solver_config(**kw):
    base = dict(dissipation_type=cb.DISS_ROE, is_second_order=1, time_accurate=1, local_time_stepping=1, cfl=0.8,
                limiter=cb.LIM_MINMOD, muscl=cb.MUSCL_GRADIENT, integrator=cb.INT_SSPRK3,
                inlet_bc=cb.INLET_TOTAL_PT, exit_bc=cb.EXIT_STATIC_P, r_gas=R_GAS, reorder=0)
    base.update(kw)
    return cb.default_config(**base)


def member_batch(meshes, params, precision=cb.PREC_FP64):
    b = cb.Batch(meshes, solver_config(precision=precision))
    bv = np.array([boundary_values(M, r) for _, M, r in params])
    inlet = np.zeros((len(meshes), 4))
    inlet[:, 0], inlet[:, 1] = bv[:, 0], bv[:, 1]
    b.set_boundary_values(inlet=inlet, exit_p=bv[:, 2])
    return b


def solve(meshes, params, states, tol, max_steps, check_every=200, r0=None, precision=cb.PREC_FP64,
          persistent=False, diverge=0.0):
    """Batched steady solves of the members from `states`, each until ||R_rho|| has dropped to
    tol * r0 (r0: given normalisers, else each member's first-step residual); returns (run
    result, final states, wall seconds).  persistent: the batch runs each RK stage as one
    persistent kernel (one CUDA graph per stage); diverge > 0: a member whose residual ratio grows
    past it stops (steps_to_tol -2)."""
    b = member_batch(meshes, params, precision)
    if persistent:
        b.set_option("persistent", 1)
    if diverge > 0.0:
        b.set_option("divergence_ratio", diverge)
    b.upload_state(states)
    if r0 is not None:
        b.set_reference_residual(r0)
    t0 = time.perf_counter()
    res = b.run(max_steps, tol, check_every)
    wall = time.perf_counter() - t0
    out = b.download_state()
    b.close()
    return res, out, wall


def solve_plain(meshes, params, states, tol, max_steps, check_every, r0):
    """The plain path: each member alone through the single-solve API, FP64, one after another,
    from its state until ||R_rho|| <= tol * r0[i] (checked every check_every pseudo-steps) or
    max_steps; returns (steps per member, -1 if not reached; final states; wall seconds)."""
    steps, out = [], []
    t0 = time.perf_counter()
    for m, (_, M, ratio), U, r in zip(meshes, params, states, r0):
        p0, T0, pe = boundary_values(M, ratio)
        s = cb.Solver(m, solver_config(inlet_p0=p0, inlet_t0=T0, exit_p=pe))
        s.set_option("keep_delu", 0)
        s.upload_state(U)
        done, k = 0, -1
        while done < max_steps:
            info = s.step(min(check_every, max_steps - done))
            done += min(check_every, max_steps - done)
            if info.res_l2[0] <= tol * r:
                k = done
                break
        steps.append(k)
        out.append(s.download_U())
        s.close()
    return np.array(steps), out, time.perf_counter() - t0


def solve_chosen(meshes, params, states, tol, max_steps, check_every, r0, switch_tol, diverge=0.0):
    """The chosen path: every member in one persistent batch; the FP32-flux form until
    ||R_rho|| <= switch_tol * r0 (its rounding floor lies near 1e-6 of the start), then the FP64
    form from that state to tol * r0.  Returns (steps per member over both phases, -1 if not
    reached, -2 if the residual grew past `diverge`; final states; wall seconds of both phases and
    the hand-over)."""
    switch_tol = max(switch_tol, tol)
    t0 = time.perf_counter()
    res1, U1, _ = solve(meshes, params, states, switch_tol, max_steps, check_every, r0=r0,
                        precision=cb.PREC_FP32_FLUX, persistent=True, diverge=diverge)
    k1 = res1["steps_to_tol"]
    grown = k1 == -2
    res2, U2, _ = solve(meshes, params, U1, tol, max_steps, check_every, r0=r0, precision=cb.PREC_FP64,
                        persistent=True, diverge=diverge)
    wall = time.perf_counter() - t0
    k2 = res2["steps_to_tol"]
    first = np.where(k1 > 0, k1, res1["steps"])
    steps = np.where(grown | (k2 == -2), -2, np.where(k2 > 0, first + k2, -1))
    return steps, U2, wall


def first_residuals(meshes, params, states):
    """||R_rho||_2 after one pseudo-step of each member from `states`."""
    b = member_batch(meshes, params)
    b.upload_state(states)
    b.run(1, 0.0, 1)
    r = b.residuals()
    b.close()
    return r


# ---------------------------------------------------------------------------------------------
# Cell graph of a member mesh
# ---------------------------------------------------------------------------------------------
class MeshGraph:
    """Directed edges between neighbouring physical cells (one per cell face with a physical
    neighbour: message from the neighbour `src` into the cell `dst`), sorted by (dst, face), with
    CSR lists by destination and by source; node and edge features of one member."""

    def __init__(self, mesh):
        NP = mesh.n_physical
        nbr = mesh.neighbours[:NP]
        dst, src, face = [], [], []
        for c in range(NP):
            for f in range(int(mesh.n_faces[c])):
                n = int(nbr[c, f])
                if 0 <= n < NP:
                    dst.append(c)
                    src.append(n)
                    face.append(f)
        self.N, self.E = NP, len(dst)
        self.dst = np.array(dst, np.int32)
        self.src = np.array(src, np.int32)
        self.face = np.array(face, np.int32)
        self.dst_ptr = np.zeros(NP + 1, np.int32)
        np.add.at(self.dst_ptr, self.dst + 1, 1)
        self.dst_ptr = np.cumsum(self.dst_ptr).astype(np.int32)
        order = np.argsort(self.src, kind="stable").astype(np.int32)
        self.src_idx = order
        self.src_ptr = np.zeros(NP + 1, np.int32)
        np.add.at(self.src_ptr, self.src + 1, 1)
        self.src_ptr = np.cumsum(self.src_ptr).astype(np.int32)

    def features(self, mesh, params):
        """Node features [N, 9]: centre (x, y), area, wall / inlet / exit face counts, and the
        member's (t, M, ratio) scaled to about [-1, 1]; edge features [E, 5]: outward normal of
        the destination cell's face, face length and centre-to-centre vector (lengths scaled by the
        mean face length)."""
        NP = self.N
        ctr = mesh.centers[:NP, :2]
        area = mesh.area[:NP]
        kinds = np.zeros((NP, 3))
        for k, c in zip(mesh.boundary[:, 0], mesh.boundary[:, 1]):
            col = {cb.BC_WALL: 0, cb.BC_INLET: 1, cb.BC_EXIT: 2}.get(int(k))
            if col is not None:
                kinds[c, col] += 1.0
        t, M, r = params
        glob = np.array([(t - 0.08) / 0.04, (M - 0.65) / 0.15, (r - 0.925) / 0.075])
        node = np.concatenate([ctr / np.array([LENGTH, HEIGHT]) * 2.0 - 1.0, (area / area.mean())[:, None] - 1.0,
                               kinds, np.broadcast_to(glob, (NP, 3))], axis=1)
        nrm = mesh.face_normals[self.dst, 2 * self.face], mesh.face_normals[self.dst, 2 * self.face + 1]
        dl = mesh.face_lengths[self.dst, self.face]
        h = dl.mean()
        d = mesh.centers[self.src, :2] - mesh.centers[self.dst, :2]
        edge = np.stack([nrm[0], nrm[1], dl / h - 1.0, d[:, 0] / h, d[:, 1] / h], axis=1)
        return node.astype(np.float32), edge.astype(np.float32)


def primitive(U):
    """(rho, u, v, p) rows of conserved rows."""
    rho = U[:, 0]
    u, v = U[:, 1] / rho, U[:, 2] / rho
    p = (GAMMA - 1.0) * (U[:, 3] - 0.5 * rho * (u * u + v * v))
    return np.stack([rho, u, v, p], axis=1)


# ---------------------------------------------------------------------------------------------
# Network: the library's kernels (csrc/mpnn_tc.cu, csrc/mpnn.cu); torch only holds device memory
# ---------------------------------------------------------------------------------------------
def _torch():
    import torch
    return torch


def _ptr(t, col=0):
    return ctypes.c_void_p(t.data_ptr() + 4 * col) if t is not None else ctypes.c_void_p(0)


def _stream(t):
    return ctypes.c_void_p(_torch().cuda.current_stream(t.device).cuda_stream)


def segment_sum(x, ptr, idx, n_rows):
    """out[r] = sum of x[idx[j]] for j in [ptr[r], ptr[r+1]) (cfd_mpnn_segment_sum)."""
    torch = _torch()
    x = x.float().contiguous()
    out = torch.empty((n_rows, x.shape[1]), dtype=torch.float32, device=x.device)
    cb._check(cb.lib().cfd_mpnn_segment_sum(_ptr(x), _ptr(ptr), _ptr(idx), n_rows, x.shape[1], _ptr(out),
                                            _stream(x)))
    return out


class GraphBatch:
    """B copies of a member graph stacked into one graph (device index arrays)."""

    def __init__(self, g, B, device):
        torch = _torch()
        N, E = g.N, g.E
        offN = (np.arange(B) * N)[:, None]
        offE = (np.arange(B) * E)[:, None]
        self.B, self.N, self.E = B, N, E
        src = (g.src[None, :] + offN).ravel()
        dst = (g.dst[None, :] + offN).ravel()
        dptr = np.concatenate([[0], (g.dst_ptr[1:][None, :] + offE).ravel()])
        sptr = np.concatenate([[0], (g.src_ptr[1:][None, :] + offE).ravel()])
        sorder = (g.src_idx[None, :] + offE).ravel()
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.int32)).to(device)
        self.src, self.dst, self.dst_ptr, self.src_ptr, self.src_order = t(src), t(dst), t(dptr), t(sptr), t(sorder)
        self.ident = t(np.arange(B * E))


def _seg(t, idx=None, col=0, width=None, silu=0):
    """One input segment: columns [col, col + width) of the rows of t (through idx when given)."""
    return (t, idx, col, t.shape[1] - col if width is None else width, silu)


class Net:
    """The message-passing surrogate: node and edge encoders, `layers` message-passing layers
    (edge update from the two end cells and the edge, in-order aggregation of each cell's incoming
    messages, node update; residual updates), a decoder; every block a two-layer perceptron
    W2 silu(W1 x + b1) + b2 of hidden width 64.  Parameters live in one FP32 device buffer (master
    copy; the kernels round operands to BF16 and accumulate in FP32); forward, backward and Adam
    are the library's kernels; torch provides device buffers only."""

    HIDDEN = 64

    def __init__(self, layers=6, node_in=9, edge_in=5, out=4, seed=0, device="cuda", engine=0, bwd_engine=None):
        torch = _torch()
        W = self.HIDDEN
        # Dense blocks: engine 0 mma.sync m16n8k16, 1 tcgen05.mma with tensor-memory accumulators
        # (forward; the backward data path follows unless bwd_engine is given).  At this network's
        # sizes (K <= 192, N <= 64) both are bound by operand staging, and 0 trains faster on B200.
        self.engine = engine
        self.bwd_engine = engine if bwd_engine is None else bwd_engine
        self.L, self.out, self.device = layers, out, torch.device(device)
        self.dims = {"enc_n": (node_in, W), "enc_e": (edge_in, W), "dec": (W, out)}
        for l in range(layers):
            self.dims["edge%d" % l] = (3 * W, W)
            self.dims["node%d" % l] = (2 * W, W)
        self.names = ["enc_n", "enc_e"] + ["edge%d" % l for l in range(layers)] + \
                     ["node%d" % l for l in range(layers)] + ["dec"]
        sizes = [W * K + W + N * W + N for K, N in (self.dims[n] for n in self.names)]
        self.n_params = int(sum(sizes))
        f32 = dict(dtype=torch.float32, device=self.device)
        self.flat = torch.zeros(self.n_params, **f32)
        self.grad = torch.zeros(self.n_params, **f32)
        self.m = torch.zeros(self.n_params, **f32)
        self.v = torch.zeros(self.n_params, **f32)
        self.p, self.g = {}, {}
        o = 0
        for name in self.names:
            K, N = self.dims[name]
            views = []
            for buf, store in ((self.flat, self.p), (self.grad, self.g)):
                q = o
                w1 = buf[q:q + W * K].view(W, K); q += W * K
                b1 = buf[q:q + W]; q += W
                w2 = buf[q:q + N * W].view(N, W); q += N * W
                b2 = buf[q:q + N]; q += N
                store[name] = (w1, b1, w2, b2)
            o = q
        rng = np.random.default_rng(seed)
        for name in self.names:
            K, N = self.dims[name]
            a, c = 1.0 / np.sqrt(K), 1.0 / np.sqrt(W)
            vals = (rng.uniform(-a, a, (W, K)), rng.uniform(-a, a, W), rng.uniform(-c, c, (N, W)), rng.uniform(-c, c, N))
            for dst, v in zip(self.p[name], vals):
                dst.copy_(torch.from_numpy(v.astype(np.float32)))
        self.workspace = torch.empty(cb.lib().cfd_mpnn_wgrad_blocks() * (W * 3 * W + W), **f32)
        self.steps = 0
        self._bufs = None

    # -- parameters as numpy (tests, checkpoints)
    def get_params(self):
        return {n: tuple(t.detach().cpu().numpy().astype(np.float64) for t in self.p[n]) for n in self.names}

    def set_params(self, P):
        torch = _torch()
        for n in self.names:
            for dst, v in zip(self.p[n], P[n]):
                dst.copy_(torch.from_numpy(np.asarray(v, np.float32)))

    def get_grads(self):
        return {n: tuple(t.detach().cpu().numpy().astype(np.float64) for t in self.g[n]) for n in self.names}

    # -- buffers per (nodes, edges)
    def _buffers(self, N, E):
        if self._bufs is not None and self._bufs["key"] == (N, E):
            return self._bufs
        torch = _torch()
        W, L = self.HIDDEN, self.L
        f = lambda r, c: torch.empty((r, c), dtype=torch.float32, device=self.device)
        b = {"key": (N, E), "h": [f(N, W) for _ in range(L + 1)], "e": [f(E, W) for _ in range(L + 1)],
             "agg": [f(N, W) for _ in range(L)], "z_enc_n": f(N, W), "z_enc_e": f(E, W),
             "z_edge": [f(E, W) for _ in range(L)], "z_node": [f(N, W) for _ in range(L)], "z_dec": f(N, W),
             "pred": f(N, self.out), "dpred": f(N, self.out), "dh": f(N, W), "de": f(E, W),
             "dx": f(max(N, E), 3 * W), "dz": f(max(N, E), W),
             "loss": torch.zeros(1, dtype=torch.float32, device=self.device)}
        self._bufs = b
        return b

    @staticmethod
    def _segs(segs):
        out = (cb.MlpSeg * 3)()
        for i, (t, idx, col, width, silu) in enumerate(segs):
            out[i].src = _ptr(t, col)
            out[i].idx = _ptr(idx) if idx is not None else ctypes.c_void_p(0)
            out[i].width, out[i].ld, out[i].silu = width, t.stride(0), silu
        return out

    def _mlp(self, name, segs, rows, y, z1, resid=None):
        a = cb.MlpFwd()
        a.rows, a.nseg, a.seg = rows, len(segs), self._segs(segs)
        w1, b1, w2, b2 = self.p[name]
        a.out = w2.shape[0]
        a.w1, a.b1, a.w2, a.b2 = _ptr(w1), _ptr(b1), _ptr(w2), _ptr(b2)
        a.resid = _ptr(resid)
        a.ld_resid = resid.stride(0) if resid is not None else 0
        a.z1, a.y, a.ld_y = _ptr(z1), _ptr(y), y.stride(0)
        a.engine = self.engine
        cb._check(cb.lib().cfd_mpnn_mlp_forward(ctypes.byref(a), _stream(y)))

    def _mlp_back(self, name, dy, z1, rows, dx=None):
        """dz1 of block `name` into the dz buffer; dx (the input gradient) when a buffer is given."""
        b = self._bufs
        w1, _, w2, _ = self.p[name]
        a = cb.MlpBwd()
        a.rows, a.in_width, a.out = rows, w1.shape[1], w2.shape[0]
        a.dy, a.ld_dy, a.z1 = _ptr(dy), dy.stride(0), _ptr(z1)
        a.w1, a.w2, a.dz1 = _ptr(w1), _ptr(w2), _ptr(b["dz"])
        a.dx, a.ld_dx = _ptr(dx), dx.stride(0) if dx is not None else 0
        a.engine = self.bwd_engine
        cb._check(cb.lib().cfd_mpnn_mlp_backward(ctypes.byref(a), _stream(dy)))

    def _wgrad(self, dz, rows, segs, dw, db):
        a = cb.MlpWgrad()
        a.rows, a.n, a.dz, a.ld_dz = rows, dw.shape[0], _ptr(dz), dz.stride(0)
        a.nseg, a.seg = len(segs), self._segs(segs)
        a.workspace, a.dw, a.db, a.accumulate = _ptr(self.workspace), _ptr(dw), _ptr(db), 0
        cb._check(cb.lib().cfd_mpnn_weight_grad(ctypes.byref(a), _stream(dz)))

    def _block_grads(self, name, dy, z1, rows, x_segs, dx=None):
        """Parameter gradients of block `name` (and dx) from its output gradient dy."""
        gw1, gb1, gw2, gb2 = self.g[name]
        self._mlp_back(name, dy, z1, rows, dx)
        self._wgrad(dy, rows, [_seg(z1, silu=1)], gw2, gb2)
        self._wgrad(self._bufs["dz"], rows, x_segs, gw1, gb1)

    def forward(self, xn, xe, gb):
        """Prediction [nodes][out] for node features xn and edge features xe (float32 device
        tensors) on the stacked graph gb; keeps the activations for backward()."""
        N, E = xn.shape[0], xe.shape[0]
        b = self._buffers(N, E)
        h, e, agg = b["h"], b["e"], b["agg"]
        self._mlp("enc_n", [_seg(xn)], N, h[0], b["z_enc_n"])
        self._mlp("enc_e", [_seg(xe)], E, e[0], b["z_enc_e"])
        lib, st = cb.lib(), _stream(xn)
        for l in range(self.L):
            self._mlp("edge%d" % l, [_seg(h[l], gb.src), _seg(h[l], gb.dst), _seg(e[l])], E, e[l + 1],
                      b["z_edge"][l], resid=e[l])
            cb._check(lib.cfd_mpnn_segment_sum_acc(_ptr(e[l + 1]), self.HIDDEN, _ptr(gb.dst_ptr), _ptr(gb.ident), N,
                                                   self.HIDDEN, _ptr(agg[l]), self.HIDDEN, 0, st))
            self._mlp("node%d" % l, [_seg(h[l]), _seg(agg[l])], N, h[l + 1], b["z_node"][l], resid=h[l])
        self._mlp("dec", [_seg(h[self.L])], N, b["pred"], b["z_dec"])
        self._graph = gb
        self._x = (xn, xe)
        return b["pred"]

    def backward(self, dpred):
        """Gradients of every parameter (into self.grad) from the prediction gradient dpred."""
        b, gb, W, L = self._bufs, self._graph, self.HIDDEN, self.L
        xn, xe = self._x
        N, E = xn.shape[0], xe.shape[0]
        lib, st = cb.lib(), _stream(dpred)
        dh, de, dx = b["dh"], b["de"], b["dx"]
        self._block_grads("dec", dpred, b["z_dec"], N, [_seg(b["h"][L])], dx=dh)
        de.zero_()
        for l in reversed(range(L)):
            h, e, agg = b["h"][l], b["e"][l], b["agg"][l]
            dxn = dx[:N, :2 * W]
            self._block_grads("node%d" % l, dh, b["z_node"][l], N, [_seg(h), _seg(agg)], dx=dxn)
            ldx = dx.stride(0)
            cb._check(lib.cfd_mpnn_add(_ptr(dh), W, _ptr(dh), W, _ptr(dxn), ldx, N, W, st))
            cb._check(lib.cfd_mpnn_gather_add(_ptr(de), W, _ptr(dxn, W), ldx, _ptr(gb.dst), E, W, st))
            dxe = dx[:E, :3 * W]
            self._block_grads("edge%d" % l, de, b["z_edge"][l], E, [_seg(h, gb.src), _seg(h, gb.dst), _seg(e)],
                              dx=dxe)
            cb._check(lib.cfd_mpnn_segment_sum_acc(_ptr(dxe), ldx, _ptr(gb.src_ptr), _ptr(gb.src_order), N, W,
                                                   _ptr(dh), W, 1, st))
            cb._check(lib.cfd_mpnn_segment_sum_acc(_ptr(dxe, W), ldx, _ptr(gb.dst_ptr), _ptr(gb.ident), N, W,
                                                   _ptr(dh), W, 1, st))
            cb._check(lib.cfd_mpnn_add(_ptr(de), W, _ptr(de), W, _ptr(dxe, 2 * W), ldx, E, W, st))
        self._block_grads("enc_e", de, b["z_enc_e"], E, [_seg(xe)])
        self._block_grads("enc_n", dh, b["z_enc_n"], N, [_seg(xn)])

    def loss_grad(self, target):
        """Mean-squared error of the last prediction against target (device scalar) and its
        gradient into the dpred buffer."""
        b = self._bufs
        n = b["pred"].numel()
        cb._check(cb.lib().cfd_mpnn_mse(_ptr(b["pred"]), _ptr(target), n, _ptr(b["dpred"]), _ptr(b["loss"]),
                                        _stream(target)))
        return b["loss"], b["dpred"]

    def adam_step(self, lr=1e-3, betas=(0.9, 0.999), eps=1e-8):
        """One Adam step over every parameter (cfd_mpnn_adam, one launch)."""
        self.steps += 1
        cb._check(cb.lib().cfd_mpnn_adam(_ptr(self.flat), _ptr(self.grad), _ptr(self.m), _ptr(self.v), self.n_params,
                                         lr, betas[0], betas[1], eps, self.steps, _stream(self.flat)))


def build_model(width=64, layers=6, node_in=9, edge_in=5, out=4, seed=0, device="cuda", engine=0):
    """The surrogate (about 187k parameters at width 64, 6 layers)."""
    assert width == Net.HIDDEN
    return Net(layers=layers, node_in=node_in, edge_in=edge_in, out=out, seed=seed, device=device, engine=engine)


def train(model, graph, node_feats, edge_feats, targets, epochs=200, batch=8, lr=1e-3, seed=0, device="cuda"):
    """Mean-squared error on the normalised (rho, u, v, p) targets, Adam; returns the per-epoch
    loss."""
    torch = _torch()
    rng = np.random.default_rng(seed)
    n = len(node_feats)
    xn = torch.from_numpy(np.stack(node_feats)).to(device)
    xe = torch.from_numpy(np.stack(edge_feats)).to(device)
    y = torch.from_numpy(np.stack(targets).astype(np.float32)).to(device)
    batches = {}
    losses = []
    for ep in range(epochs):
        perm = rng.permutation(n)
        tot = torch.zeros(1, dtype=torch.float64, device=device)
        for s in range(0, n, batch):
            idx = torch.from_numpy(perm[s:s + batch]).to(device)
            B = len(idx)
            if B not in batches:
                batches[B] = GraphBatch(graph, B, device)
            gb = batches[B]
            model.forward(xn[idx].reshape(-1, xn.shape[2]).contiguous(), xe[idx].reshape(-1, xe.shape[2]).contiguous(), gb)
            loss, dpred = model.loss_grad(y[idx].reshape(-1, 4).contiguous())
            model.backward(dpred)
            model.adam_step(lr)
            tot += loss.double() * B
        losses.append(float(tot) / n)
    return losses


def predict(model, graph, node_feats, edge_feats, batch=8, device="cuda"):
    torch = _torch()
    out = []
    for s in range(0, len(node_feats), batch):
        xn = torch.from_numpy(np.stack(node_feats[s:s + batch])).to(device)
        xe = torch.from_numpy(np.stack(edge_feats[s:s + batch])).to(device)
        gb = GraphBatch(graph, xn.shape[0], device)
        p = model.forward(xn.reshape(-1, xn.shape[2]).contiguous(), xe.reshape(-1, xe.shape[2]).contiguous(), gb)
        out.extend(p.reshape(xn.shape[0], graph.N, 4).cpu().numpy())
    return out


# ---------------------------------------------------------------------------------------------
# Experiment: train on solved members, warm-start held-out members
# ---------------------------------------------------------------------------------------------
def _with_ghosts(mesh, U_phys):
    """Full rows (ghosts copy their owner cell) from physical rows."""
    full = np.zeros((mesh.n_total, 4))
    full[:mesh.n_physical] = U_phys
    full[mesh.boundary[:, 3]] = U_phys[mesh.boundary[:, 1]]
    return full


def run_experiment(nx=64, ny=32, n_train=192, n_test=64, tol=1e-8, max_steps=400000, check_every=500, epochs=200,
                   batch=8, lr=1e-3, seed=2024, device="cuda", log=None, switch_tol=1e-5, n_plain=8, diverge=10.0,
                   engine=0):
    """The whole warm-start study; returns a dict of measured figures.

    1. Training members solved from the freestream start by the FP64 batched solver.
    2. The surrogate trained on their (rho, u, v, p) (library kernels, Adam).
    3. Held-out members: the plain path (FP64 single solves from the freestream, one after
       another; timed on the first n_plain members, the wall time per member scaled to all) and
       the chosen path (prediction, then the persistent batch in FP32-flux to switch_tol and FP64
       to tol), both to the same absolute target tol * r0 (r0: each member's first residual from
       the freestream).  Fallback, live: a prediction with a non-positive density or pressure
       starts from the freestream; a member whose residual grows past `diverge` x r0, or that
       misses the target, is solved again from the freestream (the time counts).
    4. The same batched form from the freestream start, for the gain of the prediction alone."""
    torch = _torch()
    say = log or (lambda *a: None)
    P = draw_parameters(n_train + n_test, seed)
    meshes = [make_mesh(nx, ny, t) for t, _, _ in P]
    graph = MeshGraph(meshes[0])
    feats = [graph.features(m, p) for m, p in zip(meshes, P)]
    fs_states = [freestream_state(m, M) for m, (_, M, _) in zip(meshes, P)]
    tr, te = slice(0, n_train), slice(n_train, n_train + n_test)
    out = {"mesh": "%dx%d" % (nx, ny), "cells": graph.N, "train": n_train, "test": n_test, "tol": tol,
           "switch_tol": switch_tol, "max_steps": max_steps, "epochs": epochs, "seed": seed, "n_plain": n_plain}

    # 1. Training members solved from the freestream start (the plain FP64 solver, batched).
    res_tr, U_tr, wall_tr = solve(meshes[tr], P[tr], fs_states[tr], tol, max_steps, check_every, persistent=True)
    out["train_solve_s"] = wall_tr
    out["train_converged"] = int((res_tr["steps_to_tol"] > 0).sum())
    say("train solves", wall_tr, out["train_converged"])
    targets = [primitive(U[:graph.N]) for U in U_tr]
    tgt = np.stack(targets)
    mu, sd = tgt.reshape(-1, 4).mean(0), tgt.reshape(-1, 4).std(0) + 1e-12
    norm = [((t - mu) / sd).astype(np.float32) for t in targets]

    # 2. Surrogate training.
    model = build_model(engine=engine)
    out["parameters"] = model.n_params
    out["engine"] = "tcgen05" if engine == 1 else "mma.sync"
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    losses = train(model, graph, [f[0] for f in feats[tr]], [f[1] for f in feats[tr]], norm, epochs=epochs,
                   batch=batch, lr=lr, seed=seed, device=device)
    torch.cuda.synchronize()
    out["train_s"] = time.perf_counter() - t1
    out["loss_first"], out["loss_last"] = losses[0], losses[-1]
    say("training", out["train_s"], losses[0], losses[-1])

    # 3a. Normalisers: each held-out member's first residual from the freestream.
    r0 = first_residuals(meshes[te], P[te], fs_states[te])

    # 3b. The plain path on the first n_plain members.
    npl = max(1, min(n_plain, n_test))
    k_pl, U_pl, wall_pl = solve_plain(meshes[te][:npl], P[te][:npl], fs_states[te][:npl], tol, max_steps,
                                      check_every, r0[:npl])
    out["plain_converged"] = int((k_pl > 0).sum())
    out["plain_steps_median"] = float(np.median(k_pl[k_pl > 0])) if (k_pl > 0).any() else None
    out["plain_wall_per_member_s"] = wall_pl / npl
    out["plain_wall_s"] = wall_pl / npl * n_test
    say("plain", out["plain_wall_s"], k_pl)

    # 3c. The chosen path: prediction, fallback of non-physical predictions, persistent batch.
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    pred = predict(model, graph, [f[0] for f in feats[te]], [f[1] for f in feats[te]], batch=batch, device=device)
    starts, fallback = [], np.zeros(n_test, bool)
    for i, (m, q) in enumerate(zip(meshes[te], pred)):
        q = q * sd + mu
        if not (np.all(q[:, 0] > 0) and np.all(q[:, 3] > 0)):
            fallback[i] = True
            starts.append(fs_states[n_train + i])
            continue
        starts.append(_with_ghosts(m, cb.conserved_from_primitive(q[:, 0], q[:, 1], q[:, 2], q[:, 3])))
    out["predict_s"] = time.perf_counter() - t2
    k_ch, U_ch, wall_ch = solve_chosen(meshes[te], P[te], starts, tol, max_steps, check_every, r0, switch_tol,
                                       diverge)
    redo = np.where(k_ch < 0)[0]
    wall_fb = 0.0
    if redo.size:
        # Live fallback: members whose residual grew or that missed the target, from the freestream.
        test_meshes = meshes[te]
        k_fb, U_fb, wall_fb = solve_chosen([test_meshes[i] for i in redo], P[te][redo],
                                           [fs_states[n_train + i] for i in redo], tol, max_steps, check_every,
                                           r0[redo], switch_tol)
        for j, i in enumerate(redo):
            k_ch[i] = k_fb[j]
            U_ch[i] = U_fb[j]
        fallback[redo] = True
    out["chosen_wall_s"] = out["predict_s"] + wall_ch + wall_fb
    out["chosen_converged"] = int((k_ch > 0).sum())
    out["chosen_steps_median"] = float(np.median(k_ch[k_ch > 0])) if (k_ch > 0).any() else None
    out["fallback_rate"] = float(fallback.mean())
    out["speedup_chosen_vs_plain"] = out["plain_wall_s"] / out["chosen_wall_s"]
    say("chosen", out["chosen_wall_s"], k_ch)

    # 4. The batched form from the freestream (same phases): the prediction's own gain.
    k_fs, U_fs, wall_fs = solve_chosen(meshes[te], P[te], fs_states[te], tol, max_steps, check_every, r0,
                                       switch_tol)
    ok = (k_fs > 0) & (k_ch > 0) & ~fallback
    out["batched_freestream_wall_s"] = wall_fs
    out["batched_freestream_steps_median"] = float(np.median(k_fs[k_fs > 0])) if (k_fs > 0).any() else None
    out["steps_ratio_median"] = float(np.median(k_ch[ok] / k_fs[ok])) if ok.any() else None
    out["speedup_prediction_in_batch"] = wall_fs / (out["predict_s"] + wall_ch)

    # Accuracy: prediction error and the final states of the chosen path against the plain FP64
    # solutions (the members the plain path ran) and against the batched FP64-from-freestream ones.
    pred_err = [np.linalg.norm(q * sd + mu - primitive(U_fs[i][:graph.N])) / np.linalg.norm(primitive(U_fs[i][:graph.N]))
                for i, q in enumerate(pred)]
    out["prediction_rel_l2_median"] = float(np.median(pred_err))
    out["final_state_rel_l2_vs_plain_max"] = float(max(
        np.linalg.norm(U_ch[i][:graph.N] - U_pl[i][:graph.N]) / np.linalg.norm(U_pl[i][:graph.N]) for i in range(npl)))
    out["final_state_rel_l2_vs_batched_freestream_max"] = float(max(
        np.linalg.norm(U_ch[i][:graph.N] - U_fs[i][:graph.N]) / np.linalg.norm(U_fs[i][:graph.N])
        for i in range(n_test)))
    say("warm start", out)
    return out
