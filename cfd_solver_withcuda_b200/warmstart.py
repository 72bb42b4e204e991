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
update), a decoder; width 64, SiLU, residual updates.  Dense layers run as BF16 GEMMs with FP32
accumulation (torch autocast, cuBLAS); the graph operations are the library's deterministic segment
sums (cfd_mpnn_segment_sum) and the optimiser its fused Adam step (cfd_mpnn_adam).
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


def solve(meshes, params, states, tol, max_steps, check_every=200, r0=None, precision=cb.PREC_FP64):
    """Batched steady solves of the members from `states`, each until ||R_rho|| has dropped to
    tol * r0 (r0: given normalisers, else each member's first-step residual); returns (run
    result, final states, wall seconds)."""
    b = member_batch(meshes, params, precision)
    b.upload_state(states)
    if r0 is not None:
        b.set_reference_residual(r0)
    t0 = time.perf_counter()
    res = b.run(max_steps, tol, check_every)
    wall = time.perf_counter() - t0
    out = b.download_state()
    b.close()
    return res, out, wall


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
# Network (torch: tensors, autocast GEMMs; graph operations and optimiser: library kernels)
# ---------------------------------------------------------------------------------------------
def _torch():
    import torch
    return torch


def segment_sum(x, ptr, idx, n_rows):
    """out[r] = sum of x[idx[j]] for j in [ptr[r], ptr[r+1]) (cfd_mpnn_segment_sum)."""
    torch = _torch()
    x = x.float().contiguous()
    out = torch.empty((n_rows, x.shape[1]), dtype=torch.float32, device=x.device)
    st = torch.cuda.current_stream(x.device).cuda_stream
    cb._check(cb.lib().cfd_mpnn_segment_sum(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(ptr.data_ptr()),
                                            ctypes.c_void_p(idx.data_ptr()), n_rows, x.shape[1],
                                            ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(st)))
    return out


def _functions():
    torch = _torch()

    class Gather(torch.autograd.Function):
        """Rows h[idx]; the backward pass sums the row gradients of each source row over the CSR
        list (ptr, order) of the rows that read it, in a fixed order."""

        @staticmethod
        def forward(ctx, h, idx, ptr, order):
            ctx.save_for_backward(ptr, order)
            ctx.n = h.shape[0]
            return h.index_select(0, idx.long())

        @staticmethod
        def backward(ctx, g):
            ptr, order = ctx.saved_tensors
            return segment_sum(g, ptr, order, ctx.n), None, None, None

    class Aggregate(torch.autograd.Function):
        """Sum of the incoming edge messages of each cell (edges sorted by destination)."""

        @staticmethod
        def forward(ctx, m, ptr, ident, dst):
            ctx.save_for_backward(dst)
            return segment_sum(m, ptr, ident, ptr.shape[0] - 1)

        @staticmethod
        def backward(ctx, g):
            (dst,) = ctx.saved_tensors
            return g.index_select(0, dst.long()), None, None, None

    return Gather, Aggregate


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


def build_model(width=64, layers=6, node_in=9, edge_in=5, out=4, seed=0):
    """Encoders, `layers` message-passing layers and a decoder (about 187k parameters at width 64,
    6 layers)."""
    torch = _torch()
    nn = torch.nn
    torch.manual_seed(seed)
    Gather, Aggregate = _functions()

    def mlp(i, o):
        return nn.Sequential(nn.Linear(i, width), nn.SiLU(), nn.Linear(width, o))

    class MPNN(nn.Module):
        def __init__(self):
            super().__init__()
            self.enc_n = mlp(node_in, width)
            self.enc_e = mlp(edge_in, width)
            self.edge = nn.ModuleList([mlp(3 * width, width) for _ in range(layers)])
            self.node = nn.ModuleList([mlp(2 * width, width) for _ in range(layers)])
            self.dec = mlp(width, out)

        def forward(self, xn, xe, gb):
            h = self.enc_n(xn).float()
            e = self.enc_e(xe).float()
            for fe, fn in zip(self.edge, self.node):
                hs = Gather.apply(h, gb.src, gb.src_ptr, gb.src_order)
                hd = Gather.apply(h, gb.dst, gb.dst_ptr, gb.ident)
                e = e + fe(torch.cat([hs, hd, e], dim=1)).float()
                agg = Aggregate.apply(e, gb.dst_ptr, gb.ident, gb.dst)
                h = h + fn(torch.cat([h, agg], dim=1)).float()
            return self.dec(h).float()

    return MPNN()


class Adam:
    """Adam on the model's FP32 parameters with the library's fused step (cfd_mpnn_adam)."""

    def __init__(self, params, lr=1e-3, betas=(0.9, 0.999), eps=1e-8):
        torch = _torch()
        self.params = [p for p in params if p.requires_grad]
        self.m = [torch.zeros_like(p) for p in self.params]
        self.v = [torch.zeros_like(p) for p in self.params]
        self.lr, self.b1, self.b2, self.eps, self.t = lr, betas[0], betas[1], eps, 0

    def step(self):
        torch = _torch()
        self.t += 1
        for p, m, v in zip(self.params, self.m, self.v):
            if p.grad is None:
                continue
            g = p.grad.float().contiguous()
            st = torch.cuda.current_stream(p.device).cuda_stream
            cb._check(cb.lib().cfd_mpnn_adam(ctypes.c_void_p(p.data.data_ptr()), ctypes.c_void_p(g.data_ptr()),
                                             ctypes.c_void_p(m.data_ptr()), ctypes.c_void_p(v.data_ptr()), p.numel(),
                                             self.lr, self.b1, self.b2, self.eps, self.t, ctypes.c_void_p(st)))

    def zero_grad(self):
        for p in self.params:
            p.grad = None


def train(model, graph, node_feats, edge_feats, targets, epochs=200, batch=8, lr=1e-3, seed=0, device="cuda"):
    """Mean-squared error on the normalised (rho, u, v, p) targets; returns the per-epoch loss."""
    torch = _torch()
    model.to(device)
    rng = np.random.default_rng(seed)
    n = len(node_feats)
    xn = torch.from_numpy(np.stack(node_feats)).to(device)
    xe = torch.from_numpy(np.stack(edge_feats)).to(device)
    y = torch.from_numpy(np.stack(targets).astype(np.float32)).to(device)
    opt = Adam(model.parameters(), lr=lr)
    batches = {}
    losses = []
    for ep in range(epochs):
        perm = rng.permutation(n)
        tot = 0.0
        for s in range(0, n, batch):
            idx = torch.from_numpy(perm[s:s + batch]).to(device)
            B = len(idx)
            if B not in batches:
                batches[B] = GraphBatch(graph, B, device)
            gb = batches[B]
            with torch.autocast("cuda", dtype=torch.bfloat16):
                pred = model(xn[idx].reshape(-1, xn.shape[2]), xe[idx].reshape(-1, xe.shape[2]), gb)
            loss = torch.mean((pred - y[idx].reshape(-1, 4)) ** 2)
            opt.zero_grad()
            loss.backward()
            opt.step()
            tot += float(loss.detach()) * B
        losses.append(tot / n)
    return losses


def predict(model, graph, node_feats, edge_feats, batch=8, device="cuda"):
    torch = _torch()
    out = []
    with torch.no_grad():
        for s in range(0, len(node_feats), batch):
            xn = torch.from_numpy(np.stack(node_feats[s:s + batch])).to(device)
            xe = torch.from_numpy(np.stack(edge_feats[s:s + batch])).to(device)
            gb = GraphBatch(graph, xn.shape[0], device)
            with torch.autocast("cuda", dtype=torch.bfloat16):
                p = model(xn.reshape(-1, xn.shape[2]), xe.reshape(-1, xe.shape[2]), gb)
            out.extend(p.float().reshape(xn.shape[0], graph.N, 4).cpu().numpy())
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


def run_experiment(nx=64, ny=32, n_train=192, n_test=64, tol=1e-4, max_steps=150000, check_every=500, epochs=200,
                   batch=8, lr=1e-3, seed=2024, device="cuda", log=None):
    """The whole warm-start study; returns a dict of measured figures."""
    torch = _torch()
    say = log or (lambda *a: None)
    P = draw_parameters(n_train + n_test, seed)
    meshes = [make_mesh(nx, ny, t) for t, _, _ in P]
    graph = MeshGraph(meshes[0])
    feats = [graph.features(m, p) for m, p in zip(meshes, P)]
    fs_states = [freestream_state(m, M) for m, (_, M, _) in zip(meshes, P)]
    tr, te = slice(0, n_train), slice(n_train, n_train + n_test)
    out = {"mesh": "%dx%d" % (nx, ny), "cells": graph.N, "train": n_train, "test": n_test, "tol": tol,
           "max_steps": max_steps, "epochs": epochs, "seed": seed}

    # 1. Training members solved from the freestream start (the plain FP64 solver).
    t0 = time.perf_counter()
    res_tr, U_tr, wall_tr = solve(meshes[tr], P[tr], fs_states[tr], tol, max_steps, check_every)
    out["train_solve_s"] = wall_tr
    out["train_converged"] = int((res_tr["steps_to_tol"] > 0).sum())
    say("train solves", wall_tr, out["train_converged"])
    targets = [primitive(U[:graph.N]) for U in U_tr]
    tgt = np.stack(targets)
    mu, sd = tgt.reshape(-1, 4).mean(0), tgt.reshape(-1, 4).std(0) + 1e-12
    norm = [((t - mu) / sd).astype(np.float32) for t in targets]

    # 2. Surrogate training.
    model = build_model()
    out["parameters"] = int(sum(p.numel() for p in model.parameters()))
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    losses = train(model, graph, [f[0] for f in feats[tr]], [f[1] for f in feats[tr]], norm, epochs=epochs,
                   batch=batch, lr=lr, seed=seed, device=device)
    torch.cuda.synchronize()
    out["train_s"] = time.perf_counter() - t1
    out["loss_first"], out["loss_last"] = losses[0], losses[-1]
    say("training", out["train_s"], losses[0], losses[-1])

    # 3. Held-out members from the freestream start: reference solutions and normalisers.
    r0 = first_residuals(meshes[te], P[te], fs_states[te])
    res_fs, U_fs, wall_fs = solve(meshes[te], P[te], fs_states[te], tol, max_steps, check_every, r0=r0)

    # 4. Predicted starts (denormalised; non-physical predictions fall back to freestream).
    t2 = time.perf_counter()
    pred = predict(model, graph, [f[0] for f in feats[te]], [f[1] for f in feats[te]], batch=batch, device=device)
    out["predict_s"] = time.perf_counter() - t2
    starts, fallback = [], np.zeros(n_test, bool)
    pred_err = []
    for i, (m, q) in enumerate(zip(meshes[te], pred)):
        q = q * sd + mu
        ref = primitive(U_fs[i][:graph.N])
        pred_err.append(np.linalg.norm(q - ref) / np.linalg.norm(ref))
        if not (np.all(q[:, 0] > 0) and np.all(q[:, 3] > 0)):
            fallback[i] = True
            starts.append(fs_states[n_train + i])
            continue
        starts.append(_with_ghosts(m, cb.conserved_from_primitive(q[:, 0], q[:, 1], q[:, 2], q[:, 3])))
    res_ws, U_ws, wall_ws = solve(meshes[te], P[te], starts, tol, max_steps, check_every, r0=r0)
    k_fs, k_ws = res_fs["steps_to_tol"], res_ws["steps_to_tol"]
    fallback |= (k_ws < 0) & (k_fs > 0)
    ok = (k_fs > 0) & ~fallback
    out.update({
        "freestream_converged": int((k_fs > 0).sum()), "warm_converged": int((k_ws > 0).sum()),
        "fallback_rate": float(fallback.mean()),
        "steps_freestream_median": float(np.median(k_fs[k_fs > 0])) if (k_fs > 0).any() else None,
        "steps_warm_median": float(np.median(k_ws[ok])) if ok.any() else None,
        "steps_ratio_median": float(np.median(k_ws[ok] / k_fs[ok])) if ok.any() else None,
        "wall_freestream_s": wall_fs, "wall_warm_s": wall_ws + out["predict_s"],
        "prediction_rel_l2_median": float(np.median(pred_err)),
        "final_state_rel_l2_max": float(max(np.linalg.norm(U_ws[i][:graph.N] - U_fs[i][:graph.N]) /
                                            np.linalg.norm(U_fs[i][:graph.N]) for i in range(n_test))),
    })
    say("warm start", out)
    return out
