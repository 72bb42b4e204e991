// CUDA kernels of the explicit FV residual/update path (sm_100a, FP64, --fmad=false).
//
// One thread per physical cell gathers its own faces in the reference's face order 0..nF-1,
// so every per-cell sum is formed in the same order as the reference's serial loop and the
// result is deterministic and bit-identical; there are no atomics on data.  Reductions (min dt,
// residual and error norms) use a fixed-shape warp-shuffle tree per block and a fixed-order pass
// over the per-block partials (a last-block pass, or the two-level group pass of the last stage).
#include <climits>
#include <type_traits>

#include "kernels.cuh"
#include "physics.cuh"

namespace cfdb {

namespace {

constexpr int kFluxBlock = 128;
constexpr int kFlux4Block = 128;  // 32 cells x 4 face lanes
constexpr int kBlock = 256;
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ bool step_done(const double *ctl) { return ctl[CTL_DONE] != 0.0; }

// Programmatic dependent launch: a kernel launched with programmatic stream serialization may
// start while its predecessor grid drains; it allows its own dependents to launch at entry and
// waits for the predecessor's completion (and memory) before its first global access.  Both are
// no-ops for a normal launch.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Launches kernel k (smem bytes of dynamic shared memory), with programmatic stream
// serialization when m.pdl is set and the L2 access-policy window of m when it has one.
template <typename... KArgs, typename... Args>
void launch_ks(const DevMesh &m, void (*k)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t s,
               Args... args) {
  if (!m.pdl && !m.l2_bytes) {
    k<<<grid, block, smem, s>>>(args...);
    return;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[2];
  int na = 0;
  if (m.pdl) {
    at[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[na].val.programmaticStreamSerializationAllowed = 1;
    na++;
  }
  if (m.l2_bytes) {
    at[na].id = cudaLaunchAttributeAccessPolicyWindow;
    at[na].val.accessPolicyWindow.base_ptr = m.l2_base;
    at[na].val.accessPolicyWindow.num_bytes = m.l2_bytes;
    at[na].val.accessPolicyWindow.hitRatio = m.l2_hit;
    at[na].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    at[na].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    na++;
  }
  cfg.attrs = at;
  cfg.numAttrs = na;
  cudaLaunchKernelEx(&cfg, k, args...);
}

template <typename... KArgs, typename... Args>
void launch_k(const DevMesh &m, void (*k)(KArgs...), unsigned grid, unsigned block, cudaStream_t s, Args... args) {
  launch_ks(m, k, grid, block, 0, s, args...);
}

// Item handled by this thread: from the block's work-list range when a list is given (n when the
// thread is past the range's end), else the plain global index.
__device__ __forceinline__ int item_index(const int2 *blk, int n) {
  if (blk) {
    const int2 b = blk[blockIdx.x];
    const int i = b.x + static_cast<int>(threadIdx.x);
    return i < b.y ? i : n;
  }
  return blockIdx.x * blockDim.x + threadIdx.x;
}

__device__ __forceinline__ void flag_bad(int *status, int cell) {
  atomicMin(&status[1], cell);
  atomicCAS(&status[0], 0, 3 /* CFD_ERR_NONPHYSICAL */);
}

__device__ __forceinline__ void store_prim(double *prim, double4 *q4, int NT, int c, const Prim &q) {
  prim[c] = q.rho;
  prim[NT + c] = q.u;
  prim[2 * NT + c] = q.v;
  prim[3 * NT + c] = q.p;
  prim[4 * NT + c] = q.a;
  if (q4) q4[c] = make_double4(q.rho, q.u, q.v, q.p);
}

__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double w = __shfl_xor_sync(kFull, v, o);
    v = w < v ? w : v;
  }
  return v;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// Block-wide min; result valid in thread 0.
__device__ __forceinline__ double block_min(double v, double *sh) {
  v = warp_min(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    v = lane < nw ? sh[lane] : 1e308 * 10.0;
    v = warp_min(v);
  }
  return v;
}

// Block-wide sum (fixed tree); result valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double *sh) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    v = lane < nw ? sh[lane] : 0.0;
    v = warp_sum(v);
  }
  return v;
}

// Warp sums of 8 per-lane values in 9 shuffles: three halving exchanges leave each lane one
// quantity q = 4*bit4 + 2*bit3 + bit2 of its lane id summed over 8 lanes, two more sum the 4
// lanes that share it.  Fixed order, so deterministic.
__device__ __forceinline__ double warp_sums8(const double v[8], int &q) {
  const int lane = threadIdx.x & 31;
  const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4;
  double a[4], b[2];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const double send = h16 ? v[i] : v[i + 4], keep = h16 ? v[i + 4] : v[i];
    a[i] = keep + __shfl_xor_sync(kFull, send, 16);
  }
#pragma unroll
  for (int i = 0; i < 2; i++) {
    const double send = h8 ? a[i] : a[i + 2], keep = h8 ? a[i + 2] : a[i];
    b[i] = keep + __shfl_xor_sync(kFull, send, 8);
  }
  const double send = h4 ? b[0] : b[1], keep = h4 ? b[1] : b[0];
  double c = keep + __shfl_xor_sync(kFull, send, 4);
  c += __shfl_xor_sync(kFull, c, 2);
  c += __shfl_xor_sync(kFull, c, 1);
  q = (h16 ? 4 : 0) + (h8 ? 2 : 0) + (h4 ? 1 : 0);
  return c;
}

// Block sums of 8 per-thread values; the sum of quantity q is returned in thread q (q < 8).
__device__ __forceinline__ double block_sums8(const double v[8], double *sh /* 8 * 32 */) {
  int q;
  const double c = warp_sums8(v, q);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if ((lane & 3) == 0) sh[q * 32 + w] = c;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x < 8)
    for (int i = 0; i < nw; i++) s += sh[threadIdx.x * 32 + i];
  return s;
}

// Final sums over the per-block partials partial[q * nb + i] (q < NQ), run by the last block: one
// warp per quantity, each lane over a fixed stride of blocks, then a shuffle tree.  The sum of q
// is returned in lane 0 of warp q % (warps per block) for the iteration that handled q.
template <int NQ, typename Store>
__device__ __forceinline__ void sum_partials(const double *partial, int nb, Store store) {
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int q = threadIdx.x >> 5; q < NQ; q += nw) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    const double *p = partial + (size_t)q * nb;
    int i = lane;
    for (; i + 96 < nb; i += 128) {
      a0 += __ldcg(p + i);
      a1 += __ldcg(p + i + 32);
      a2 += __ldcg(p + i + 64);
      a3 += __ldcg(p + i + 96);
    }
    for (; i < nb; i += 32) a0 += __ldcg(p + i);
    double a = warp_sum((a0 + a1) + (a2 + a3));
    if (lane == 0) store(q, a);
  }
}

// Reduces nq quantities of n values each, src[q * stride + i] for i < n: the minimum for quantity
// 0 when has_min, sums otherwise.  Warp w takes quantities w, w + nw, ... (at most 3 per warp);
// every lane issues its strided loads of all its quantities before any arithmetic, then a fixed
// shuffle tree, so the result is deterministic.  store(q, v) runs in lane 0 of q's warp.
template <typename Store>
__device__ __forceinline__ void reduce_rows(const double *src, int stride, int n, int nq, bool has_min, Store store) {
  constexpr int kMaxQ = 3, kPer = 4;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const double kInf = 1e308 * 10.0;
  int qs[kMaxQ];
  double acc[kMaxQ];
#pragma unroll
  for (int j = 0; j < kMaxQ; j++) {
    qs[j] = w + j * nw;
    acc[j] = (has_min && qs[j] == 0) ? kInf : 0.0;
  }
  for (int base = 0; base < n; base += 32 * kPer) {
    double v[kMaxQ][kPer];
#pragma unroll
    for (int j = 0; j < kMaxQ; j++)
#pragma unroll
      for (int k = 0; k < kPer; k++) {
        const int i = base + k * 32 + lane;
        const bool mn = has_min && qs[j] == 0;
        v[j][k] = (qs[j] < nq && i < n) ? __ldcg(src + (size_t)qs[j] * stride + i) : (mn ? kInf : 0.0);
      }
#pragma unroll
    for (int j = 0; j < kMaxQ; j++)
#pragma unroll
      for (int k = 0; k < kPer; k++) {
        if (has_min && qs[j] == 0) acc[j] = v[j][k] < acc[j] ? v[j][k] : acc[j];
        else acc[j] += v[j][k];
      }
  }
#pragma unroll
  for (int j = 0; j < kMaxQ; j++) {
    if (qs[j] >= nq) continue;  // uniform across the warp
    const double r = (has_min && qs[j] == 0) ? warp_min(acc[j]) : warp_sum(acc[j]);
    if (lane == 0) store(qs[j], r);
  }
}

// Returns true in every thread of the block that finished last among the grid's blocks.  The
// only data the last block reads from other blocks are their partials, which every caller writes
// from threads of warp 0; only that warp fences (a fence in every warp would hold each warp until
// all of its state stores were acknowledged).
__device__ __forceinline__ bool last_block(unsigned int *counter) {
  __shared__ bool is_last;
  if (threadIdx.x < 32) __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned t = atomicAdd(counter, 1u);
    is_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  return is_last;
}

// Two-level grid reduction of 9 per-block values, written at partial[q * nb + blockIdx.x] by
// threads of warp 0 (q = 0: a minimum, q = 1..8: sums).  Blocks form groups of G consecutive
// blocks; the last block of a group to finish reduces the group's partials in block order into
// partial[9 nb + q * ngroups + group], and the last group to finish reduces those in group order
// into out[9] (shared memory).  Both rounds are a single set of independent loads, and the group
// rounds run while other blocks are still working.  Returns true in the block that wrote out.
__device__ __forceinline__ bool grid_reduce9(DevState &st, double *out) {
  __shared__ bool flag;
  const int nb = gridDim.x;
  const int G = max(32, (nb + kMaxGroups - 1) / kMaxGroups);
  const int ngroups = (nb + G - 1) / G;
  const int grp = blockIdx.x / G;
  const int gsize = min(G, nb - grp * G);
  if (threadIdx.x < 32) __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) flag = (atomicAdd(&st.gcount[grp], 1u) == (unsigned)(gsize - 1));
  __syncthreads();
  if (!flag) return false;
  double *gp = st.partial + 9 * (size_t)nb;
  reduce_rows(st.partial + (size_t)grp * G, nb, gsize, 9, true,
              [&](int q, double v) { gp[(size_t)q * ngroups + grp] = v; });
  if (threadIdx.x == 0) st.gcount[grp] = 0u;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) flag = (atomicAdd(&st.gcount[kMaxGroups], 1u) == (unsigned)(ngroups - 1));
  __syncthreads();
  if (!flag) return false;
  reduce_rows(gp, ngroups, ngroups, 9, true, [&](int q, double v) { out[q] = v; });
  if (threadIdx.x == 0) st.gcount[kMaxGroups] = 0u;
  __syncthreads();
  return true;
}

// ---------------------------------------------------------------------------------------------
__global__ void k_prim_all(DevMesh m, DevState st) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.NT) return;
  const double *U = st.U;
  Prim q;
  bool ok = eos_prim(U[c], U[m.NT + c], U[2 * m.NT + c], U[3 * m.NT + c], q);
  store_prim(st.prim, st.q4, m.NT, c, q);
  if (!ok) flag_bad(st.status, c);
}

// Apply_Boundary_Conditions (src/Boundary_Conditions.cpp:12-61): one thread per
// (kind, cell, face, ghost) entry writes U and primitives of the ghost row.
//   wall / symmetry  src/Wall_Boundary_Conditions.cpp:8-53, :79-124 (reflect V about the face normal)
//   supersonic inlet src/Inlet_Boundary_Conditions.cpp:41-74 (rho, p prescribed, V extrapolated)
//   subsonic inlet   src/Inlet_Boundary_Conditions.cpp:7-39 (reference energy form)
//   supersonic exit  src/Exit_Boundary_Conditions.cpp:68-94 (copy of U_Cells of the interior cell)
//   subsonic exit    src/Exit_Boundary_Conditions.cpp:83-85 (no-op in the reference)
// Additive forms: total-(p, T) characteristic inflow and static-pressure outflow.
//   far field        CUDA_KERNELS/Boundary_Conditions_Cuda_Kernels.cu:257-325 (inlet kind 4)
//   fixed-p exit     src/Exit_Boundary_Conditions.cpp:8-66 (exit kind 3)
// src_is_S: the supersonic-exit copy reads the stage state (stage-consistent forms) instead of
// U^n; cur_is_S: the state the primitives were last computed from is the stage state.
__device__ __forceinline__ void bc_entry(const DevMesh &m, DevState &st, const BcParams &bp, int e, int src_is_S,
                                         int cur_is_S) {
  const int4 b = m.bnd[e];
  const int kind = b.x, c = b.y, f = b.z, g = b.w;
  const int NT = m.NT, NP = m.NP;
  const double *prim = st.prim;
  const double rho = prim[c], u = prim[NT + c], v = prim[2 * NT + c], p = prim[3 * NT + c];
  double G0, G1, G2, G3;
  if (kind == 2 || kind == 3) {
    const double n1 = m.nx[f * NP + c], n2 = m.ny[f * NP + c];
    double vdotn = (u * n1 + v * n2);
    double v1g = u - 2.0 * vdotn * n1;
    double v2g = v - 2.0 * vdotn * n2;
    double vmag = 0.5 * (v1g * v1g + v2g * v2g);
    G0 = rho;
    G1 = rho * v1g;
    G2 = rho * v2g;
    G3 = ((p / kGM1) + rho * vmag);
  } else if (kind == 0) {
    if (bp.inlet_bc == 4) {
      const double *Uc = cur_is_S ? st.S : st.U;
      const int ld = cur_is_S ? NP : NT;
      const double Ui[4] = {Uc[c], Uc[ld + c], Uc[2 * ld + c], Uc[3 * ld + c]};
      double Gf[4];
      const double4 fs = m.bstate ? m.bstate[e] : make_double4(bp.inlet_rho, bp.inlet_u, bp.inlet_v, bp.inlet_p);
      farfield_state(Ui, m.nx[f * NP + c], m.ny[f * NP + c], fs.x, fs.y, fs.z, fs.w, Gf);
      G0 = Gf[0];
      G1 = Gf[1];
      G2 = Gf[2];
      G3 = Gf[3];
    } else if (bp.inlet_bc == 3) {
      // Fully prescribed inflow (rho, u, v, p), per boundary entry when given (batched solves).
      const double4 q = m.bstate ? m.bstate[e] : make_double4(bp.inlet_rho, bp.inlet_u, bp.inlet_v, bp.inlet_p);
      G0 = q.x;
      G1 = q.x * q.y;
      G2 = q.x * q.z;
      G3 = q.w / kGM1 + 0.5 * q.x * (q.y * q.y + q.z * q.z);
    } else if (bp.inlet_bc == 0) {
      double vmag = (u * u + v * v) * 0.5;
      G0 = bp.inlet_rho;
      G1 = bp.inlet_rho * u;
      G2 = bp.inlet_rho * v;
      G3 = (bp.inlet_p / kGM1) + bp.inlet_rho * vmag;
    } else if (bp.inlet_bc == 1) {
      double Vm = 0.5 * (u * u + v * v);
      G0 = bp.inlet_rho;
      G1 = bp.inlet_rho * u;
      G2 = bp.inlet_rho * v;
      G3 = (bp.inlet_p / kGM1) + bp.inlet_rho * Vm * Vm;
    } else {
      // Subsonic inflow with total pressure p0 and total temperature T0 (no reference
      // counterpart: the reference's subsonic inlet is the form above).  n is the outward
      // normal, so inflow has Vn < 0 and the characteristic Vn + a leaves the domain: its
      // invariant R+ = Vn + 2a/(g-1) comes from the interior.  With V = Vn n and
      // H0 = a0^2/(g-1) = a^2/(g-1) + Vn^2/2 this gives
      //   (g+1)/(g-1) a^2 - 2 R+ a + (g-1)/2 R+^2 - a0^2 = 0   (larger root),
      // then Vn = R+ - 2a/(g-1), T = a^2/(g R), p = p0 (T/T0)^(g/(g-1)), rho = p/(R T).
      const double n1 = m.nx[f * NP + c], n2 = m.ny[f * NP + c];
      const double a_i = prim[4 * NT + c];
      const double vn_i = u * n1 + v * n2;
      const double Rp = vn_i + 2.0 * a_i / kGM1;
      const double p0 = m.bstate ? m.bstate[e].x : bp.inlet_p0, t0 = m.bstate ? m.bstate[e].y : bp.inlet_t0;
      const double a0sq = kGamma * bp.r_gas * t0;
      const double qa = (kGamma + 1.0) / kGM1, qb = -2.0 * Rp, qc = 0.5 * kGM1 * Rp * Rp - a0sq;
      const double disc = qb * qb - 4.0 * qa * qc;
      const double ab = (-qb + sqrt(disc > 0.0 ? disc : 0.0)) / (2.0 * qa);
      double vn = Rp - 2.0 * ab / kGM1;
      if (vn > 0.0) vn = 0.0;
      const double Tb = ab * ab / (kGamma * bp.r_gas);
      const double pb = p0 * pow(Tb / t0, kGamma / kGM1);
      const double rb = pb / (bp.r_gas * Tb);
      const double ub = vn * n1, vb = vn * n2;
      G0 = rb;
      G1 = rb * ub;
      G2 = rb * vb;
      G3 = pb / kGM1 + 0.5 * rb * (ub * ub + vb * vb);
    }
  } else {  // exit
    if (bp.exit_bc == 1) return;
    const double *Us = src_is_S ? st.S : st.U;
    const int ld = src_is_S ? NP : NT;
    if (bp.exit_bc == 0) {
      G0 = Us[c];
      G1 = Us[ld + c];
      G2 = Us[2 * ld + c];
      G3 = Us[3 * ld + c];
    } else if (bp.exit_bc == 3) {
      const double rho_Et = cur_is_S ? st.S[3 * NP + c] : st.U[3 * NT + c];
      double Gf[4];
      fixed_p_exit_state(rho, u, v, p, rho_Et, m.nx[f * NP + c], m.ny[f * NP + c], m.bexit ? m.bexit[e] : bp.exit_p,
                         Gf);
      G0 = Gf[0];
      G1 = Gf[1];
      G2 = Gf[2];
      G3 = Gf[3];
    } else {
      // Static-pressure outflow: rho, V extrapolated; p prescribed when the normal Mach
      // number is subsonic, extrapolated otherwise.
      const double n1 = m.nx[f * NP + c], n2 = m.ny[f * NP + c];
      const double a_i = prim[4 * NT + c];
      const double vn = u * n1 + v * n2;
      const double pb = (vn < a_i) ? (m.bexit ? m.bexit[e] : bp.exit_p) : p;
      G0 = rho;
      G1 = rho * u;
      G2 = rho * v;
      G3 = pb / kGM1 + 0.5 * rho * (u * u + v * v);
    }
  }
  double *U = st.U;
  U[g] = G0;
  U[NT + g] = G1;
  U[2 * NT + g] = G2;
  U[3 * NT + g] = G3;
  Prim q;
  bool ok = eos_prim(G0, G1, G2, G3, q);
  store_prim(st.prim, st.q4, NT, g, q);
  if (!ok) flag_bad(st.status, g);
}

__global__ void k_bc(DevMesh m, DevState st, BcParams bp, int src_is_S, int cur_is_S) {
  pdl_enter();
  const int e = item_index(m.bblk, m.NB);
  if (e >= m.NB || step_done(st.ctl)) return;
  bc_entry(m, st, bp, e, src_is_S, cur_is_S);
}

// Conserved state of cell n for the limiter / LLF: U_Cells (U^n on physical rows, boundary
// values on ghost rows) in the reference's semantics, or the current stage state.
struct USrc {
  const double *U, *S;
  int NT, NP, use_S;
  __device__ __forceinline__ double get(int k, int n) const {
    return (use_S && n < NP) ? S[k * NP + n] : U[k * NT + n];
  }
};

// The state of the cell whose faces are being evaluated.
struct CellState {
  double rc, uc, vc, pc, ac;
  double Uc[4];
  uint8_t degen;
};

template <int DISS, int ORDER>
__device__ __forceinline__ void load_cell(const DevMesh &m, const DevState &st, const USrc &us, int c, CellState &q) {
  const int NT = m.NT;
  const double *prim = st.prim;
  q.rc = prim[c];
  q.uc = prim[NT + c];
  q.vc = prim[2 * NT + c];
  q.pc = prim[3 * NT + c];
  q.ac = prim[4 * NT + c];
  if (DISS == 1 || DISS == 2 || DISS == 5 || DISS == 6 || DISS == 7 || ORDER == 2) {
#pragma unroll
    for (int k = 0; k < 4; k++) q.Uc[k] = us.get(k, c);
  }
  q.degen = m.degen[c];
}

// Contribution of face f of cell c: X = avg - diss (Calculate_Flux_For_All_Faces,
// src/Net_Flux.cpp:18-43) and the del_t term (|V.n| + a) dl (src/Time_Step.cpp:326-336).
template <int DISS, int ORDER>
__device__ __forceinline__ void face_contrib(const DevMesh &m, const DevState &st, const FluxParams &fp,
                                             const USrc &us, const CellState &q, int c, int f, double X[4],
                                             double &t) {
  const int NP = m.NP, NT = m.NT;
  const double *prim = st.prim;
  const double rc = q.rc, uc = q.uc, vc = q.vc, pc = q.pc, ac = q.ac;
  const int idx = f * NP + c;
  const int N = m.nbr[idx];
  const double nx = m.nx[idx], ny = m.ny[idx], dl = m.dl[idx];
  const double rn = prim[N], un = prim[NT + N], vn = prim[2 * NT + N], pn = prim[3 * NT + N], an = prim[4 * NT + N];
  double A[4], D[4];
  if (DISS != 6 && DISS != 7) average_flux<double>(rc, uc, vc, pc, rn, un, vn, pn, nx, ny, dl, A);
  if (DISS == 3 && ORDER == 1) {
    if (N >= NP)
      roe_1o<double>(rc, uc, vc, pc, ac, rc, uc, vc, pc, ac, nx, ny, dl, (q.degen >> f) & 1, D);
    else
      roe_1o<double>(rc, uc, vc, pc, ac, rn, un, vn, pn, an, nx, ny, dl, (q.degen >> f) & 1, D);
  } else if (DISS == 3 && ORDER == 2) {
    const int n2 = m.n2[idx];
    const double d1 = m.d1l[idx], d2 = m.d2l[idx];
    double dU[4];
    if (!fp.recon_prim) {
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const double q1 = us.get(k, N), q2 = us.get(k, n2);
        const double phi = limited_slope<double>(fp.limiter, q.Uc[k], q1, q2, d1, d2, fp.zeta, fp.zeta1);
        const double VR = q1 + 0.5 * phi * d1;
        const double VL = q.Uc[k] - 0.5 * phi * d1;
        dU[k] = VR - VL;
      }
    } else {
      // MUSCL on (rho, u, v, p) of the stage primitives on the reference stencil; the
      // conserved jump of the two reconstructed face states drives the Roe wave strengths.
      const double qc[4] = {rc, uc, vc, pc};
      const double q1v[4] = {rn, un, vn, pn};
      const double q2v[4] = {prim[n2], prim[NT + n2], prim[2 * NT + n2], prim[3 * NT + n2]};
      double qR[4], qL[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const double phi = limited_slope<double>(fp.limiter, qc[k], q1v[k], q2v[k], d1, d2, fp.zeta, fp.zeta1);
        qR[k] = q1v[k] + 0.5 * phi * d1;
        qL[k] = qc[k] - 0.5 * phi * d1;
      }
      dU[0] = qR[0] - qL[0];
      dU[1] = qR[0] * qR[1] - qL[0] * qL[1];
      dU[2] = qR[0] * qR[2] - qL[0] * qL[2];
      dU[3] = (qR[3] / kGM1 + 0.5 * qR[0] * (qR[1] * qR[1] + qR[2] * qR[2])) -
              (qL[3] / kGM1 + 0.5 * qL[0] * (qL[1] * qL[1] + qL[2] * qL[2]));
    }
    roe_2o<double>(rc, uc, vc, pc, ac, rn, un, vn, pn, an, nx, ny, dl, dU, D);
  } else if (DISS == 2 || DISS == 4 || DISS == 5) {
    // MOVERS, RICCA, MOVERS_NWSC and their second-order forms (src/MOVERS.cpp, src/RICCA.cpp,
    // src/MOVERS_NWSC.cpp); RICCA_2O and MOVERS_NWSC_2O take the limited conserved jump of
    // Second_Order_Limiter (src/Limiters.cpp:97-200), MOVERS_2O does not call it.
    double UR[4], dU2[4] = {0.0, 0.0, 0.0, 0.0};
    if (DISS != 4 || ORDER == 2) {
#pragma unroll
      for (int k = 0; k < 4; k++) UR[k] = us.get(k, N);
    }
    if (ORDER == 2 && DISS != 2) {
      const int n2 = m.n2[idx];
      const double d1 = m.d1l[idx], d2 = m.d2l[idx];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const double q2 = us.get(k, n2);
        const double phi = limited_slope<double>(fp.limiter, q.Uc[k], UR[k], q2, d1, d2, fp.zeta, fp.zeta1);
        const double VR = UR[k] + 0.5 * phi * d1;
        const double VL = q.Uc[k] - 0.5 * phi * d1;
        dU2[k] = VR - VL;
      }
    }
    if (DISS == 2)
      movers_diss<double, ORDER>(rc, uc, vc, pc, ac, rn, un, vn, pn, an, q.Uc, UR, nx, ny, dl, fp.movers_single,
                                 fp.movers_efix, D);
    else if (DISS == 4)
      ricca_diss<double, ORDER>(rc, uc, vc, pc, rn, un, vn, pn, nx, ny, dl, dU2, D);
    else
      nwsc_diss<double, ORDER>(rc, uc, vc, pc, rn, un, vn, pn, q.Uc, UR, nx, ny, dl, dU2, D);
  } else if (DISS == 6 || DISS == 7) {
    // Reference forms of AUSM (src/Ausm_Flux.cpp:26-34, from U_Cells) and HLLC
    // (CUDA_KERNELS/HLLC_LLF_Flux_Cuda_Kernels.cu:98-100): faces whose neighbour is a ghost are
    // skipped; the net flux is the sum of the face fluxes.
#pragma unroll
    for (int k = 0; k < 4; k++) A[k] = D[k] = 0.0;
    if (N < NP) {
      double UR[4];
#pragma unroll
      for (int k = 0; k < 4; k++) UR[k] = us.get(k, N);
      if (DISS == 6) {
        ausm_face<double>(q.Uc, UR, nx, ny, dl, A);
      } else {
        const double qL[5] = {rc, uc, vc, pc, ac}, qR[5] = {rn, un, vn, pn, an};
        hllc_face<double>(qL, q.Uc, qR, UR, nx, ny, dl, A);
      }
    }
  } else {  // LLF 1O
    double UR[4];
#pragma unroll
    for (int k = 0; k < 4; k++) UR[k] = us.get(k, N);
    llf_1o<double>(uc, vc, ac, un, vn, an, q.Uc, UR, nx, ny, dl, D);
  }
#pragma unroll
  for (int k = 0; k < 4; k++) X[k] = A[k] - D[k];
  const double vnf = uc * nx + vc * ny;
  t = (fabs(vnf) + ac) * dl;
}

// del_t = CFL * Area / sum (|V.n| + a) dl, 0 when the sum is not a positive finite number
// (Inviscid_Time_Step, src/Time_Step.cpp:337-358).
__device__ __forceinline__ double cell_dt_a(const FluxParams &fp, double area, double den) {
  if (den <= 0.0 || !isfinite(den)) return 0.0;
  return fp.cfl * area / den;
}
__device__ __forceinline__ double cell_dt(const DevMesh &m, const FluxParams &fp, int c, double den) {
  return cell_dt_a(fp, m.area[c], den);
}

// Block min of del_t to `partial`; the last block writes Min_dt (get_Min_dt,
// src/Numerical_Method.cpp:322-330).
__device__ __forceinline__ void min_dt_epilogue(DevState &st, double dt, double *sh) {
  double bm = block_min(dt, sh);
  if (threadIdx.x == 0) st.partial[blockIdx.x] = bm;
  if (last_block(st.counter)) {
    double v = 1e308 * 10.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
      double w = __ldcg(&st.partial[i]);
      v = w < v ? w : v;
    }
    v = block_min(v, sh);
    if (threadIdx.x == 0) {
      st.ctl[CTL_DTMIN] = v;
      *st.counter = 0u;
    }
  }
}

// Evaluate_Cell_Net_Flux_1O/2O (src/Net_Flux.cpp:46-129) + Evaluate_Time_Step (src/Time_Step.cpp:293-359)
// fused, one thread per cell: faces in order, Net += avg - diss; then del_t; block min + Min_dt.
// MINB: minimum resident blocks per SM the register allocation is made for (1: unconstrained;
// the second-order forms with the directional limiter are also built for 6 and 8, which cap
// their 114 - 124 registers at 80 and 64 for more resident warps; the autotuner picks, the
// results are the same bits).  SRC_S false: the conserved states come from U only (the caller
// knows no stage state is read), which saves the per-load choice between U and the stage state.
template <int DISS, int ORDER, int MINB = 1, bool SRC_S = true>
__global__ void __launch_bounds__(kFluxBlock, MINB) k_flux(DevMesh m, DevState st, FluxParams fp, int src_is_S) {
  __shared__ double sh[32];
  const int NP = m.NP, NT = m.NT;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const bool done = step_done(st.ctl);
  double dt = 1e308 * 10.0;
  if (c < NP && !done) {
    const USrc us{st.U, st.S, NT, NP, SRC_S && fp.consistent && src_is_S};
    CellState q;
    load_cell<DISS, ORDER>(m, st, us, c, q);
    const int nf = m.nf[c];
    double N0 = 0.0, N1s = 0.0, N2s = 0.0, N3s = 0.0;
    double den = 0.0;
#pragma unroll
    for (int f = 0; f < 4; f++) {
      if (f < nf) {
        double X[4], t;
        face_contrib<DISS, ORDER>(m, st, fp, us, q, c, f, X, t);
        N0 += X[0];
        N1s += X[1];
        N2s += X[2];
        N3s += X[3];
        den += t;
      }
    }
    dt = cell_dt(m, fp, c, den);
    st.R[c] = N0;
    st.R[NP + c] = N1s;
    st.R[2 * NP + c] = N2s;
    st.R[3 * NP + c] = N3s;
    st.dtc[c] = dt;
  }
  if (done) return;
  min_dt_epilogue(st, dt, sh);
}

// The same evaluation with four lanes per cell (one face each): lane 0 of each quad adds the
// quad's face contributions in face order 0..nF-1 (warp shuffles), so every sum keeps the
// reference's order and value; fewer live registers per thread give the SM more warps to hide
// the gather and FP64 latencies.
template <int DISS, int ORDER>
__global__ void __launch_bounds__(kFlux4Block) k_flux4(DevMesh m, DevState st, FluxParams fp, int src_is_S) {
  __shared__ double sh[32];
  const int NP = m.NP, NT = m.NT;
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = gid >> 2, f = gid & 3;
  const bool done = step_done(st.ctl);
  if (done) return;
  const bool cell_ok = c < NP;
  const int nf = cell_ok ? m.nf[c] : 0;
  double X[4] = {0.0, 0.0, 0.0, 0.0}, t = 0.0;
  if (f < nf) {
    const USrc us{st.U, st.S, NT, NP, fp.consistent && src_is_S};
    CellState q;
    load_cell<DISS, ORDER>(m, st, us, c, q);
    face_contrib<DISS, ORDER>(m, st, fp, us, q, c, f, X, t);
  }
  double Y[3][4], T[3];
#pragma unroll
  for (int d = 1; d < 4; d++) {
#pragma unroll
    for (int k = 0; k < 4; k++) Y[d - 1][k] = __shfl_down_sync(kFull, X[k], d, 4);
    T[d - 1] = __shfl_down_sync(kFull, t, d, 4);
  }
  double dt = 1e308 * 10.0;
  if (cell_ok && f == 0) {
    double R[4] = {0.0, 0.0, 0.0, 0.0};
    double den = 0.0;
#pragma unroll
    for (int k = 0; k < 4; k++) R[k] += X[k];
    den += t;
#pragma unroll
    for (int d = 1; d < 4; d++) {
      if (d < nf) {
#pragma unroll
        for (int k = 0; k < 4; k++) R[k] += Y[d - 1][k];
        den += T[d - 1];
      }
    }
    dt = cell_dt(m, fp, c, den);
#pragma unroll
    for (int k = 0; k < 4; k++) st.R[k * NP + c] = R[k];
    st.dtc[c] = dt;
  }
  min_dt_epilogue(st, dt, sh);
}

// Evaluate_Cell_Net_Flux_WENO, src/WENO2D.cpp:395-456, one thread per cell.  Quad cells only
// (others get a zero net flux and their del_t, as in the reference).  Stencils walk the neighbour
// slots as the reference does (WENO_Reconstruction_X, :245-393): slot 0 / 1 for the "i" walks and
// 2 / 3 for the "j" walks, a ghost repeated when the walk leaves the domain.  The stencil values
// are the conserved variables the reference rebuilds from the primitives
// (Calculate_Computational_Variables, src/Basic_Functions.cpp:156-163): rho, rho*u, rho*v and the
// energy the primitives were computed from (cur_is_S: the stage state for physical cells).
__device__ __forceinline__ void weno_cons(const DevMesh &m, const DevState &st, int i, int cur_is_S, double U[4]) {
  const int NP = m.NP, NT = m.NT;
  const double rho = st.prim[i];
  U[0] = rho;
  U[1] = rho * st.prim[NT + i];
  U[2] = rho * st.prim[2 * NT + i];
  U[3] = (i < NP && cur_is_S) ? st.S[3 * NP + i] : st.U[3 * NT + i];
}

// Get_Reconstructed_U, src/WENO2D.cpp:216-243.
__device__ __forceinline__ bool weno_recon(const DevMesh &m, const DevState &st, int cur_is_S, bool chr,
                                           const double Lm[16], const double ILm[16], int i1, int i2, int i3, int i4,
                                           int i5, int lr, double U[4]) {
  double s[5][4];
  weno_cons(m, st, i1, cur_is_S, s[0]);
  weno_cons(m, st, i2, cur_is_S, s[1]);
  weno_cons(m, st, i3, cur_is_S, s[2]);
  weno_cons(m, st, i4, cur_is_S, s[3]);
  weno_cons(m, st, i5, cur_is_S, s[4]);
  if (chr) {
    double w[5][4], W[4];
#pragma unroll
    for (int k = 0; k < 5; k++) weno_matvec(Lm, s[k], w[k]);
#pragma unroll
    for (int i = 0; i < 4; i++) W[i] = weno5(w[0][i], w[1][i], w[2][i], w[3][i], w[4][i], lr);
    weno_matvec(ILm, W, U);
  } else {
#pragma unroll
    for (int i = 0; i < 4; i++) U[i] = weno5(s[0][i], s[1][i], s[2][i], s[3][i], s[4][i], lr);
  }
  return true;
}

__global__ void __launch_bounds__(kFluxBlock) k_weno(DevMesh m, DevState st, FluxParams fp, int cur_is_S) {
  __shared__ double sh[32];
  const int NP = m.NP, NT = m.NT;
  const int c = item_index(m.cblk, NP);
  const bool done = step_done(st.ctl);
  double dt = 1e308 * 10.0;
  if (c < NP && !done) {
    const int nf = m.nf[c];
    double R[4] = {0.0, 0.0, 0.0, 0.0};
    bool ok = true;
    if (nf == 4) {
      const int im1 = m.nbr[c], ip1 = m.nbr[NP + c], jm1 = m.nbr[2 * NP + c], jp1 = m.nbr[3 * NP + c];
      int im2, im3, ip2, ip3, jm2, jm3, jp2, jp3;
      if (im1 >= NP) {
        im2 = im1;
        im3 = im1;
      } else {
        im2 = m.nbr[im1];
        if (im2 >= NP || im2 < 0) {
          im3 = im2;
        } else {
          im3 = m.nbr[im2];
          if (im3 < 0) im3 = im2;
        }
      }
      if (ip1 >= NP) {
        ip2 = ip1;
        ip3 = ip1;
      } else {
        ip2 = m.nbr[NP + ip1];
        if (ip2 >= NP || ip2 < 0) {
          ip3 = ip2;
        } else {
          ip3 = m.nbr[NP + ip2];
          if (ip3 < 0) ip3 = ip2;
        }
      }
      if (jm1 >= NP) {
        jm2 = jm1;
        jm3 = jm1;
      } else {
        jm2 = m.nbr[2 * NP + jm1];
        jm3 = (jm2 >= NP) ? jm2 : m.nbr[2 * NP + jm2];
      }
      if (jp1 >= NP) {
        jp2 = jp1;
        jp3 = jp1;
      } else {
        jp2 = m.nbr[3 * NP + jp1];
        jp3 = (jp2 >= NP) ? jp2 : m.nbr[3 * NP + jp2];
      }
      // Face stencils (left: shift 0, right: shift 1) of WENO_Reconstruction_X's switch.
      const int st5[4][2][5] = {{{im3, im2, im1, c, ip1}, {im2, im1, c, ip1, ip2}},
                                {{jm3, jm2, jm1, c, jp1}, {jm2, jm1, c, jp1, jp2}},
                                {{im2, im1, c, ip1, ip2}, {im1, c, ip1, ip2, ip3}},
                                {{jm2, jm1, c, jp1, jp2}, {jm1, c, jp1, jp2, jp3}}};
      const int nb[4] = {im1, ip1, jm1, jp1};
#pragma unroll 1
      for (int f = 0; f < 4; f++) {
        const int idx = f * NP + c;
        const double nx = m.nx[idx], ny = m.ny[idx], dl = m.dl[idx];
        double Lm[16], ILm[16];
        if (fp.weno_char) {
          const int N = nb[f];
          ok = weno_lr(st.prim[c], st.prim[NT + c], st.prim[2 * NT + c], st.prim[4 * NT + c], st.prim[N],
                       st.prim[NT + N], st.prim[2 * NT + N], st.prim[4 * NT + N], nx, ny, Lm, ILm) && ok;
        }
        double UL[4], UR[4], F[4];
        const int *a = st5[f][0], *b = st5[f][1];
        weno_recon(m, st, cur_is_S, fp.weno_char, Lm, ILm, a[0], a[1], a[2], a[3], a[4], 0, UL);
        weno_recon(m, st, cur_is_S, fp.weno_char, Lm, ILm, b[0], b[1], b[2], b[3], b[4], 1, UR);
        ok = weno_face_flux(UL, UR, nx, ny, dl, F) && ok;
#pragma unroll
        for (int k = 0; k < 4; k++) R[k] += F[k];
      }
    }
    if (!ok) flag_bad(st.status, c);
    // Evaluate_Time_Step (src/Time_Step.cpp:293-329) from the cell's own state.
    const double uc = st.prim[NT + c], vc = st.prim[2 * NT + c], ac = st.prim[4 * NT + c];
    double den = 0.0;
    for (int f = 0; f < nf; f++) {
      const int idx = f * NP + c;
      const double vnf = uc * m.nx[idx] + vc * m.ny[idx];
      den += (fabs(vnf) + ac) * m.dl[idx];
    }
    dt = cell_dt(m, fp, c, den);
#pragma unroll
    for (int k = 0; k < 4; k++) st.R[k * NP + c] = R[k];
    st.dtc[c] = dt;
  }
  min_dt_epilogue(st, dt, sh);
}

// Face-based evaluation (the Green-Gauss-gradient MUSCL form; no reference counterpart): one
// thread per unique face computes the flux once from its owner's side, in precision T (double,
// or float for the FP32-flux form); the neighbour receives exactly the negated flux, so the
// scheme is conservative to the last bit.  MUSCL on (rho, u, v, p): with d = x_N - x_c and
// D+ = q_N - q_c, the upwind differences are D-_c = 2 grad q_c . d - D+ and
// D-_N = 2 grad q_N . d - D+; q_L = q_c + 0.5 phi(D-_c, D+) D+, q_R = q_N - 0.5 phi(D-_N, D+) D+
// (phi(a, b), r = a/b; the product phi D+ evaluated as muscl_slope).  A ghost neighbour uses the owner's gradient.  A non-positive
// reconstructed density or pressure falls back to the cell-centre state.  Flux: average of the two
// face states plus Roe dissipation between them (with the linear-wave entropy fix when
// fp.eflin > 0).
// Flux of one unique face from the owner's record (c0: rho, u, v, p; c1, c2: gradients) and the
// neighbour's (n0, n1, n2), face normal (nx, ny), length dl and centre-to-centre vector (dx, dy).
template <typename T, int DISS>
__device__ __forceinline__ double4 face_flux_rec(int glim, const double4 c0, const double4 c1, const double4 c2,
                                                 const double4 n0, const double4 n1, const double4 n2, const T nx,
                                                 const T ny, const T dl, const T dx, const T dy, const T eflin,
                                                 const T shock_fix = T(0.0)) {
  const T qc[4] = {T(c0.x), T(c0.y), T(c0.z), T(c0.w)};
  const T qn[4] = {T(n0.x), T(n0.y), T(n0.z), T(n0.w)};
  const T gc[8] = {T(c1.x), T(c1.y), T(c1.z), T(c1.w), T(c2.x), T(c2.y), T(c2.z), T(c2.w)};
  const T gn[8] = {T(n1.x), T(n1.y), T(n1.z), T(n1.w), T(n2.x), T(n2.y), T(n2.z), T(n2.w)};
  T qL[4], qR[4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const T dp = qn[k] - qc[k];
    const T dmc = T(2.0) * (gc[2 * k] * dx + gc[2 * k + 1] * dy) - dp;
    const T dmn = T(2.0) * (gn[2 * k] * dx + gn[2 * k + 1] * dy) - dp;
    qL[k] = qc[k] + T(0.5) * muscl_slope<T>(glim, dmc, dp);
    qR[k] = qn[k] - T(0.5) * muscl_slope<T>(glim, dmn, dp);
  }
  if (!(qL[0] > T(0.0)) || !(qL[3] > T(0.0))) {
#pragma unroll
    for (int k = 0; k < 4; k++) qL[k] = qc[k];
  }
  if (!(qR[0] > T(0.0)) || !(qR[3] > T(0.0))) {
#pragma unroll
    for (int k = 0; k < 4; k++) qR[k] = qn[k];
  }
  const T aL = sqrt(T(kGamma) * qL[3] / qL[0]), aR = sqrt(T(kGamma) * qR[3] / qR[0]);
  T A[4], D[4] = {T(0.0), T(0.0), T(0.0), T(0.0)};
  // DISS 3: Roe; DISS 103: Roe with the options of the form (linear-wave entropy fix, shock-stable
  // hybrid), a separate instance so that the plain form keeps its register footprint.
  if (DISS == 3 || DISS == 103) {
    average_flux<T>(qL[0], qL[1], qL[2], qL[3], qR[0], qR[1], qR[2], qR[3], nx, ny, dl, A);
    // Shock sensor of the hybrid: |grad p|^2 |d|^2 > (shock_fix p)^2 in either cell.
    bool rusanov = false;
    if (DISS == 103 && shock_fix > T(0.0)) {
      const T d2 = dx * dx + dy * dy;
      const T gpc = gc[6] * gc[6] + gc[7] * gc[7], gpn = gn[6] * gn[6] + gn[7] * gn[7];
      const T tc = shock_fix * qc[3], tn = shock_fix * qn[3];
      rusanov = gpc * d2 > tc * tc || gpn * d2 > tn * tn;
    }
    if (rusanov) {
      const T vnL = qL[1] * nx + qL[2] * ny, vnR = qR[1] * nx + qR[2] * ny;
      const T sL = fabs(vnL) + aL, sR = fabs(vnR) + aR;
      const T sm = sL > sR ? sL : sR;
      const T UL[4] = {qL[0], qL[0] * qL[1], qL[0] * qL[2],
                       qL[3] / T(kGM1) + T(0.5) * qL[0] * (qL[1] * qL[1] + qL[2] * qL[2])};
      const T UR[4] = {qR[0], qR[0] * qR[1], qR[0] * qR[2],
                       qR[3] / T(kGM1) + T(0.5) * qR[0] * (qR[1] * qR[1] + qR[2] * qR[2])};
#pragma unroll
      for (int k = 0; k < 4; k++) D[k] = T(0.5) * sm * (UR[k] - UL[k]) * dl;
    } else {
      roe_1o<T>(qL[0], qL[1], qL[2], qL[3], aL, qR[0], qR[1], qR[2], qR[3], aR, nx, ny, dl, false, D,
                DISS == 103 ? eflin : T(0.0));
    }
  } else {
    // Conserved face states for AUSM / HLLC: E = p/(g-1) + rho |V|^2 / 2.
    const T UL[4] = {qL[0], qL[0] * qL[1], qL[0] * qL[2],
                     qL[3] / T(kGM1) + T(0.5) * qL[0] * (qL[1] * qL[1] + qL[2] * qL[2])};
    const T UR[4] = {qR[0], qR[0] * qR[1], qR[0] * qR[2],
                     qR[3] / T(kGM1) + T(0.5) * qR[0] * (qR[1] * qR[1] + qR[2] * qR[2])};
    if (DISS == 6) {
      ausm_face<T>(UL, UR, nx, ny, dl, A);
    } else if (DISS == 8) {
      ausm_gpu_face<T>(UL, UR, nx, ny, dl, A);
    } else {
      const T q5L[5] = {qL[0], qL[1], qL[2], qL[3], aL}, q5R[5] = {qR[0], qR[1], qR[2], qR[3], aR};
      hllc_face<T>(q5L, UL, q5R, UR, nx, ny, dl, A);
    }
  }
  return make_double4(double(A[0] - D[0]), double(A[1] - D[1]), double(A[2] - D[2]), double(A[3] - D[3]));
}

template <typename T, int DISS, int MINB>
__global__ void __launch_bounds__(MINB >= 6 ? 128 : 256, MINB) k_faces(DevMesh m, DevState st, FluxParams fp) {
  pdl_enter();
  const int i = item_index(m.fblk, m.NF);
  if (i >= m.NF || step_done(st.ctl)) return;
  const int NP = m.NP;
  const int2 on = m.fon[i];
  const int c = on.x, N = on.y;
  const int glim = fp.limiter == LIM_REF_MINMOD ? LIM_MINMOD : fp.limiter;
  const double4 gq = m.fg4[i];
  const T nx = T(gq.x), ny = T(gq.y), dl = T(gq.z), dx = T(gq.w), dy = T(m.fdy[i]);
  const double4 c0 = st.q4[c], n0 = st.q4[N];
  const bool nphys = N < NP;
  double4 c1, c2, n1, n2;
  if (sizeof(T) == sizeof(float)) {
    // FP32-flux form: 32-byte float records (the values face_flux_rec would round to anyway).
    const float4 *rc = st.recf + 2 * (size_t)c, *rn = st.recf + 2 * (size_t)N;
    const float4 a = rc[0], b = rc[1];
    c1 = make_double4(a.x, a.y, a.z, a.w);
    c2 = make_double4(b.x, b.y, b.z, b.w);
    if (nphys) {
      const float4 p = rn[0], q = rn[1];
      n1 = make_double4(p.x, p.y, p.z, p.w);
      n2 = make_double4(q.x, q.y, q.z, q.w);
    } else {
      n1 = c1;
      n2 = c2;
    }
  } else {
    const double4 *rc = reinterpret_cast<const double4 *>(st.rec + 8 * (size_t)c);
    const double4 *rn = reinterpret_cast<const double4 *>(st.rec + 8 * (size_t)N);
    c1 = rc[0];
    c2 = rc[1];
    n1 = nphys ? rn[0] : c1;
    n2 = nphys ? rn[1] : c2;
  }
  st.F[i] = face_flux_rec<T, DISS>(glim, c0, c1, c2, n0, n1, n2, nx, ny, dl, dx, dy, T(fp.eflin),
                                     T(fp.shock_fix));
}

// Sum of the face fluxes of cell c in face order (+F on the owner side, -F on the neighbour
// side) and the del_t denominator.  The cell's four face-table slots come in one 16-byte load
// without waiting for the face count (an unused slot holds face 0), so the flux loads of every
// face are in flight together; only the sums are predicated on the count.
// CG: the face fluxes were written earlier in the same launch by other thread blocks (the
// persistent stage kernel), so they are loaded from L2 (ld.global.cg), not through L1.
__device__ __forceinline__ double4 ldcg4(const double4 *p) {
  const double2 a = __ldcg(reinterpret_cast<const double2 *>(p));
  const double2 b = __ldcg(reinterpret_cast<const double2 *>(p) + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

template <bool DEN = true, bool CG = false>
__device__ __forceinline__ void gather_faces(const DevMesh &m, const DevState &st, int c, double R[4], double &den) {
  const int NP = m.NP, NT = m.NT;
  const double uc = DEN ? st.prim[NT + c] : 0.0, vc = DEN ? st.prim[2 * NT + c] : 0.0,
               ac = DEN ? st.prim[4 * NT + c] : 0.0;
  const int nf = m.nf[c];
  const int4 e4 = m.cface4[c];
  const int e[4] = {e4.x, e4.y, e4.z, e4.w};
  double4 F[4];
#pragma unroll
  for (int f = 0; f < 4; f++) {
    const int id = e[f] < 0 ? -e[f] - 1 : e[f];
    F[f] = CG ? ldcg4(st.F + id) : st.F[id];
  }
  R[0] = R[1] = R[2] = R[3] = 0.0;
  den = 0.0;
#pragma unroll
  for (int f = 0; f < 4; f++) {
    if (f < nf) {
      if (e[f] < 0) {
        R[0] += -F[f].x;
        R[1] += -F[f].y;
        R[2] += -F[f].z;
        R[3] += -F[f].w;
      } else {
        R[0] += F[f].x;
        R[1] += F[f].y;
        R[2] += F[f].z;
        R[3] += F[f].w;
      }
      if (DEN) {
        const int idx = f * NP + c;
        const double vnf = uc * m.nx[idx] + vc * m.ny[idx];
        den += (fabs(vnf) + ac) * m.dl[idx];
      }
    }
  }
}

// Per cell: Net = sum of its face fluxes in face order, del_t from the cell's own state
// (src/Time_Step.cpp:293-329), block min.
__global__ void __launch_bounds__(kFluxBlock) k_gather(DevMesh m, DevState st, FluxParams fp) {
  __shared__ double sh[32];
  const int NP = m.NP;
  const int c = item_index(m.cblk, NP);
  const bool done = step_done(st.ctl);
  double dt = 1e308 * 10.0;
  if (c < NP && !done) {
    double R[4], den;
    gather_faces(m, st, c, R, den);
    dt = cell_dt(m, fp, c, den);
#pragma unroll
    for (int k = 0; k < 4; k++) st.R[k * NP + c] = R[k];
    st.dtc[c] = dt;
  }
  if (done) return;
  min_dt_epilogue(st, dt, sh);
}

// Estimate_Error (src/Error_Estimate_Update.cpp:10-28) terms of one cell; dU < 1e-9 is the
// reference's signed test.
__device__ __forceinline__ double err_term(double du, double u) {
  double t;
  if (du < 1e-9) t = fabs(du);
  else t = fabs(du) / u;
  return t * t;
}

// Per-block partial sums (4 error terms, 4 residual squares), then the last block reduces the
// partials in block order and applies the step epilogue (Total_Time += Min_dt, iterations++).
__device__ __forceinline__ void reduce_err_and_epilogue(DevState &st, const double e[8], bool advance_time,
                                                        double dt_for_time) {
  __shared__ double sh[8 * 32];
  double v[8];
#pragma unroll
  for (int q = 0; q < 8; q++) v[q] = e[q];
  const double s = block_sums8(v, sh);
  if (threadIdx.x < 8) st.partial[threadIdx.x * gridDim.x + blockIdx.x] = s;
  if (last_block(st.counter)) {
    double *ctl = st.ctl;
    sum_partials<8>(st.partial, (int)gridDim.x,
                    [ctl](int q, double a) { ctl[(q < 4 ? CTL_ERR + q : CTL_RES + q - 4)] = sqrt(a); });
    __syncthreads();
    if (threadIdx.x == 0) {
      if (advance_time) {
        double t = st.ctl[CTL_TOTAL_TIME] + dt_for_time;
        st.ctl[CTL_TOTAL_TIME] = t;
        st.ctl[CTL_ITER] += 1.0;
        double te = st.ctl[CTL_TEND];
        if (te > 0.0 && t >= te) st.ctl[CTL_DONE] = 1.0;
      }
      *st.counter = 0u;
    }
  }
}

// Stage updates of Runge_Kutta_Method (src/Numerical_Method.cpp:342-457) and Explicit_Method
// (:26-103) for one cell, written with the reference's association order.  kind: 1,2,3 RK3
// stages, 0 explicit, 11..14 classical RK4.  The final kind writes dU and, with fuse_final,
// applies Estimate_Error's terms (e[0..3]), the residual squares (e[4..7]) and Update().
// Stage kinds: 0 explicit; 1-3 the three-stage forms (reference Runge_Kutta_Method or SSP-RK3);
// 11-14 classical RK4; 21-23 the reference GPU TVD-RK3 kernel (21, 22 equal 1, 2); 31-34 the
// reference GPU RK4 kernel.  Kinds 23 and 34 produce U^{n+1} itself, the others dU.
__host__ __device__ __forceinline__ bool first_kind(int kind) {
  return kind == 1 || kind == 11 || kind == 21 || kind == 31;
}
__host__ __device__ __forceinline__ bool final_kind(int kind) {
  return kind == 0 || kind == 3 || kind == 14 || kind == 23 || kind == 34;
}
__host__ __device__ __forceinline__ bool direct_kind(int kind) { return kind == 23 || kind == 34; }

// Inputs of one cell's stage update that do not depend on the residual: U^n, the stage state
// (RK3 stages 2 and 3) and 1/A.  Loaded ahead of the residual gather so that both sets of loads
// are in flight together.
struct StageIn {
  double Un[4], Sk[4], invA;
};

__device__ __forceinline__ void load_stage_in(const DevMesh &m, const DevState &st, int c, int kind, StageIn &in) {
  const int NP = m.NP, NT = m.NT;
  in.invA = m.inv_area[c];
#pragma unroll
  for (int k = 0; k < 4; k++) in.Un[k] = st.U[k * NT + c];
  if (kind == 2 || kind == 3 || kind == 22 || kind == 23) {
#pragma unroll
    for (int k = 0; k < 4; k++) in.Sk[k] = st.S[k * NP + c];
  }
}

__device__ __forceinline__ void cell_update_in(const DevMesh &m, DevState &st, int c, int kind, double dt,
                                               const double Rk[4], const StageIn &in, int fuse_final, int keep_delu,
                                               double e[8]) {
  const int NP = m.NP, NT = m.NT;
  const double invA = in.invA;
  double Un[4], out[4];
#pragma unroll
  for (int k = 0; k < 4; k++) Un[k] = in.Un[k];
  bool final_stage = false;
  if (kind == 1 || kind == 21) {
#pragma unroll
    for (int k = 0; k < 4; k++) out[k] = Un[k] - dt * invA * Rk[k];
  } else if (kind == 2 || kind == 22) {
#pragma unroll
    for (int k = 0; k < 4; k++) out[k] = 0.25 * (in.Sk[k] + 3.0 * Un[k] - dt * invA * Rk[k]);
  } else if (kind == 3) {
#pragma unroll
    for (int k = 0; k < 4; k++) out[k] = (2.0 / 3.0) * (in.Sk[k] - Un[k] - dt * invA * Rk[k]);
    final_stage = true;
  } else if (kind == 0) {
#pragma unroll
    for (int k = 0; k < 4; k++) out[k] = -dt * invA * Rk[k];
    final_stage = true;
  } else if (kind == 23) {
    // tvd_rk3_kernel stage 3 (CUDA_KERNELS/Time_Integration_Cuda_Kernels.cu:125-130):
    // U^{n+1} = (1/3)(U^n + 2 U2 - 2 dt/V R(U2)).
#pragma unroll
    for (int k = 0; k < 4; k++) out[k] = (1.0 / 3.0) * (Un[k] + 2.0 * in.Sk[k] - 2.0 * dt * invA * Rk[k]);
    final_stage = true;
  } else if (kind == 31 || kind == 32) {
    // rk4_complete_kernel stages 1-2 (CUDA_KERNELS/Time_Integration_Cuda_Kernels.cu:43-56): the
    // stage state is U^n - dt/(2V) R of the previous stage state (its dissipation terms are zero
    // for the inviscid path).
#pragma unroll
    for (int k = 0; k < 4; k++) out[k] = Un[k] - 0.5 * dt * invA * Rk[k];
  } else if (kind == 33) {
#pragma unroll
    for (int k = 0; k < 4; k++) out[k] = Un[k] - dt * invA * Rk[k];
  } else if (kind == 34) {
    // Stage 4 (:64-72): U^{n+1} = U^n - dt/(6V) R(U3), the last stage's residual only.
#pragma unroll
    for (int k = 0; k < 4; k++) out[k] = Un[k] - (dt * invA / 6.0) * Rk[k];
    final_stage = true;
  } else if (kind == 11) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      st.Racc[k * NP + c] = Rk[k];
      out[k] = Un[k] - 0.5 * (dt * invA) * Rk[k];
    }
  } else if (kind == 12 || kind == 13) {
    const double w = (kind == 12) ? 0.5 : 1.0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      st.Racc[k * NP + c] = st.Racc[k * NP + c] + 2.0 * Rk[k];
      out[k] = Un[k] - w * (dt * invA) * Rk[k];
    }
  } else {  // 14
#pragma unroll
    for (int k = 0; k < 4; k++) {
      double acc = st.Racc[k * NP + c] + Rk[k];
      out[k] = -((dt * invA) * acc) / 6.0;
    }
    final_stage = true;
  }
  if (!final_stage) {
#pragma unroll
    for (int k = 0; k < 4; k++) st.S[k * NP + c] = out[k];
    Prim q;
    bool ok = eos_prim(out[0], out[1], out[2], out[3], q);
    store_prim(st.prim, st.q4, NT, c, q);
    if (!ok) flag_bad(st.status, c);
  } else {
    // dU and U^{n+1}: the forms that produce U^{n+1} directly keep it exactly (dU = U^{n+1} - U^n
    // is stored for Estimate_Error, and U^{n+1} is parked in the stage state for Update()).
    const bool direct = direct_kind(kind);
    double du[4], nu[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      du[k] = direct ? out[k] - Un[k] : out[k];
      nu[k] = direct ? out[k] : Un[k] + out[k];
    }
    if (keep_delu || !fuse_final) {
#pragma unroll
      for (int k = 0; k < 4; k++) st.dU[k * NP + c] = du[k];
    }
    if (direct && !fuse_final) {
#pragma unroll
      for (int k = 0; k < 4; k++) st.S[k * NP + c] = nu[k];
    }
    if (fuse_final) {
#pragma unroll
      for (int k = 0; k < 4; k++) {
        e[k] += err_term(du[k], Un[k]);  // callers start e at 0 (strided callers sum their cells)
        e[4 + k] += Rk[k] * Rk[k];
        st.U[k * NT + c] = nu[k];
        Un[k] = nu[k];
      }
      Prim q;
      bool ok = eos_prim(Un[0], Un[1], Un[2], Un[3], q);
      store_prim(st.prim, st.q4, NT, c, q);
      if (!ok) flag_bad(st.status, c);
    }
  }
}

__device__ __forceinline__ void cell_update(const DevMesh &m, DevState &st, int c, int kind, double dt,
                                            const double Rk[4], int fuse_final, int keep_delu, double e[8]) {
  StageIn in;
  load_stage_in(m, st, c, kind, in);
  cell_update_in(m, st, c, kind, dt, Rk, in, fuse_final, keep_delu, e);
}

// lts: 0 Min_dt, 1 Cell::del_t (reference stage 1 only), 2 dt frozen per cell at the first stage,
// 3 Min_dt frozen at the first stage.
__global__ void __launch_bounds__(kBlock) k_stage(DevMesh m, DevState st, int kind, int lts, int fuse_final,
                                                  int keep_delu) {
  const int NP = m.NP;
  const int c = item_index(m.cblk, NP);
  const bool done = step_done(st.ctl);
  const bool active = c < NP && !done;
  double e[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const double dtmin = st.ctl[CTL_DTMIN];
  if (active) {
    const bool first = first_kind(kind);
    if (first) {
      if (lts == 2) st.dtk[c] = st.dtc[c];
    }
    double dt;
    if (lts == 0) dt = dtmin;
    else if (lts == 1) dt = st.dtc[c];
    else if (lts == 2) dt = first ? st.dtc[c] : st.dtk[c];
    else dt = first ? dtmin : st.ctl[CTL_DTSTEP];
    double Rk[4];
#pragma unroll
    for (int k = 0; k < 4; k++) Rk[k] = st.R[k * NP + c];
    cell_update(m, st, c, kind, dt, Rk, fuse_final, keep_delu, e);
  }
  if (first_kind(kind) && blockIdx.x == 0 && threadIdx.x == 0 && !done) st.ctl[CTL_DTSTEP] = dtmin;
  if (fuse_final && final_kind(kind)) {
    if (done) return;
    const double dt_time = (lts >= 2) ? st.ctl[CTL_DTSTEP] : dtmin;
    reduce_err_and_epilogue(st, e, true, dt_time);
  }
}

// Stage update of cell c from its residual R, shared by the gather and patch forms: stores R,
// takes the stage dt (lts 1: del_t of this evaluation; else del_t frozen at the first stage),
// updates the cell, and with flags bit 1 writes the next stage's ghost states from the owner
// thread (every ghost depends only on its owner cell's new state: Apply_Boundary_Conditions of the
// next stage).  Returns the dt used.
// stage_cell_in: the same with the stage inputs and the frozen dt already loaded (the TMA tile
// form prefetches them into shared memory).
__device__ __forceinline__ double stage_cell_in(const DevMesh &m, DevState &st, const BcParams &bp, int c,
                                                const double R[4], double dtc, double dt_frozen, const StageIn &in,
                                                int kind, int lts, int fuse_final, int keep_delu, int flags,
                                                double e[8]) {
  const int NP = m.NP;
  const bool first = first_kind(kind);
#pragma unroll
  for (int k = 0; k < 4; k++) st.R[k * NP + c] = R[k];
  double dt;
  if (lts == 1) dt = dtc;
  else {
    if (first) st.dtk[c] = dtc;
    dt = first ? dtc : dt_frozen;
  }
  cell_update_in(m, st, c, kind, dt, R, in, fuse_final, keep_delu, e);
  if ((flags & 2) && !final_kind(kind)) {
    const int b0 = m.bptr[c], b1 = m.bptr[c + 1];
    for (int i = b0; i < b1; i++) bc_entry(m, st, bp, m.bidx[i], (flags & 4) ? 1 : 0, 1);
  }
  return dt;
}
__device__ __forceinline__ double stage_cell(const DevMesh &m, DevState &st, const BcParams &bp, int c,
                                             const double R[4], double dtc, int kind, int lts, int fuse_final,
                                             int keep_delu, int flags, double e[8]) {
  StageIn in;
  load_stage_in(m, st, c, kind, in);
  const double dt_frozen = (lts != 1 && !first_kind(kind)) ? st.dtk[c] : 0.0;
  return stage_cell_in(m, st, bp, c, R, dtc, dt_frozen, in, kind, lts, fuse_final, keep_delu, flags, e);
}

// Last stage of the fused forms: Estimate_Error's terms, the residual squares and the step's dt
// (the minimum of the per-cell dt frozen at the first stage, i.e. that stage's Min_dt), reduced
// over the grid, then the Total_Time epilogue of the loop body.  Called by every thread.
// stage_final_reduce_sm: the same with its scratch (32 + 8 * 32 + 9 doubles) in caller-provided
// shared memory.
__device__ __forceinline__ void stage_final_reduce_sm(DevState &st, const double e[8], double dtu, double *scratch) {
  double *sh = scratch, *sh8 = scratch + 32, *red = scratch + 32 + 8 * 32;
  const double sq = block_sums8(e, sh8);
  if (threadIdx.x < 8) st.partial[(1 + threadIdx.x) * gridDim.x + blockIdx.x] = sq;
  const double bm = block_min(dtu, sh);
  if (threadIdx.x == 0) st.partial[blockIdx.x] = bm;
  if (grid_reduce9(st, red) && threadIdx.x == 0) {
    st.ctl[CTL_DTMIN] = red[0];
    st.ctl[CTL_DTSTEP] = red[0];
    for (int q = 0; q < 8; q++) st.ctl[q < 4 ? CTL_ERR + q : CTL_RES + q - 4] = sqrt(red[1 + q]);
    double t = st.ctl[CTL_TOTAL_TIME] + red[0];
    st.ctl[CTL_TOTAL_TIME] = t;
    st.ctl[CTL_ITER] += 1.0;
    double te = st.ctl[CTL_TEND];
    if (te > 0.0 && t >= te) st.ctl[CTL_DONE] = 1.0;
  }
}
__device__ __forceinline__ void stage_final_reduce(DevState &st, const double e[8], double dtu) {
  __shared__ double scratch[32 + 8 * 32 + 9];
  stage_final_reduce_sm(st, e, dtu, scratch);
}

// Face-based forms with a per-cell time step (lts 1 or 2): the gather of k_gather and the stage
// update of k_stage in one pass, so the residual never leaves registers on its way to the update
// (it is still stored for downloads).  At the final stage the error norms, the step's Min_dt and
// the Total_Time epilogue.
// 80 registers (6 blocks of 128 per SM, 24 warps) without spilling; the unbounded build takes 84
// (5 blocks) and measured 9 % slower on B200.
// STRIDED (the reducing last stage without work lists): a grid of one wave strides over the
// cells, so the per-block fence and arrival count of the grid reduction is paid once per resident
// block instead of once per 128 cells; each thread sums its cells' terms in cell order and the
// grid is fixed per device, so the sums are reproducible.  Its accumulators spill 64 bytes at the
// same 80-register cap, which measured faster than 96 registers at 5 blocks per SM.
template <bool STRIDED>
__global__ void __launch_bounds__(kFluxBlock, 6) k_gather_stage(DevMesh m, DevState st, FluxParams fp,
                                                                             BcParams bp, int kind, int lts,
                                                                             int fuse_final, int keep_delu, int flags) {
  pdl_enter();
  const int NP = m.NP;
  if (step_done(st.ctl)) return;
  double dtu = 1e308 * 10.0;
  double e[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (!STRIDED) {
    const int c = item_index(m.cblk, NP);
    if (c < NP) {
      // The residual gather is issued first; loading the state rows ahead of it (more registers,
      // fewer resident warps) measured slower on B200.
      double R[4], den = 0.0;
      gather_faces<false>(m, st, c, R, den);
      const double dtc = (lts == 1 || first_kind(kind)) ? st.dtc[c] : 0.0;  // the only stages that use it
      dtu = stage_cell(m, st, bp, c, R, dtc, kind, lts, fuse_final, keep_delu, flags, e);
    }
  } else {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < NP; c += gridDim.x * blockDim.x) {
      double R[4], den = 0.0;
      gather_faces<false>(m, st, c, R, den);
      const double dtc = (lts == 1 || first_kind(kind)) ? st.dtc[c] : 0.0;
      const double dt = stage_cell(m, st, bp, c, R, dtc, kind, lts, fuse_final, keep_delu, flags, e);
      dtu = dt < dtu ? dt : dtu;
    }
  }
  if (fuse_final && final_kind(kind)) stage_final_reduce(st, e, dtu);
}

// Estimate_Error alone (src/Error_Estimate_Update.cpp:10-28).
__global__ void __launch_bounds__(kBlock) k_error(DevMesh m, DevState st) {
  const int NP = m.NP, NT = m.NT;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  double e[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (c < NP) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      e[k] = err_term(st.dU[k * NP + c], st.U[k * NT + c]);
      double r = st.R[k * NP + c];
      e[4 + k] = r * r;
    }
  }
  reduce_err_and_epilogue(st, e, false, 0.0);
}

// Update() (src/Error_Estimate_Update.cpp:31-43): U += dU, primitives refreshed.
// from_S: the integrator produced U^{n+1} itself (reference GPU forms), parked in the stage state.
__global__ void __launch_bounds__(kBlock) k_update(DevMesh m, DevState st, int from_S) {
  const int NP = m.NP, NT = m.NT;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= NP) return;
  double u[4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    u[k] = from_S ? st.S[k * NP + c] : st.U[k * NT + c] + st.dU[k * NP + c];
    st.U[k * NT + c] = u[k];
  }
  Prim q;
  bool ok = eos_prim(u[0], u[1], u[2], u[3], q);
  store_prim(st.prim, st.q4, NT, c, q);
  if (!ok) flag_bad(st.status, c);
}

// Calculate_Gradient_At_Cell_Center (src/Grid_Refine_Functions.cpp:221-246); var indexes the
// device primitive planes (0 rho, 1 u, 2 v, 3 p, 4 a).
__device__ __forceinline__ void gg_gradient(const DevMesh &m, const double *q, int c, double &g0, double &g1) {
  g0 = 0.0;
  g1 = 0.0;
  const int nf = m.nf[c];
  if (nf <= 0 || m.area[c] <= 0.0) return;
  const double pc = q[c];
  for (int f = 0; f < nf; f++) {
    const int idx = f * m.NP + c;
    const int N = m.nbr[idx];
    double pn = pc;
    if (N >= 0 && N < m.NP) pn = q[N];
    const double pf = 0.5 * (pc + pn);
    g0 += pf * m.nx[idx] * m.dl[idx];
    g1 += pf * m.ny[idx] * m.dl[idx];
  }
  g0 *= m.inv_area[c];
  g1 *= m.inv_area[c];
}

// Green-Gauss gradients of (rho, u, v, p) of physical cell c from the primitive planes `prim`
// ([5][NT]), multiplied by 1/A (g[2k], g[2k+1]: d/dx, d/dy of variable k), and with DT the
// denominator of del_t (Inviscid_Time_Step, src/Time_Step.cpp:293-329, faces in order).  The
// four neighbour slots come in one 16-byte load without waiting for the face count (an unused
// slot reads the cell itself), so every neighbour's loads are in flight together; the sums run
// over the cell's faces in order.
// q4 is not __restrict__: the first-stage gradient pass writes the ghost rows it then reads.
template <bool DT, bool Q4 = false>
__device__ __forceinline__ void cell_gradients(const DevMesh &m, const double *prim, const double4 *q4, int c,
                                               const double qc[4], double g[8], double &den) {
  const int NP = m.NP, NT = m.NT;
  const int nf = m.nf[c];
  const double ia = m.inv_area[c];
  const double ac = DT ? prim[4 * NT + c] : 0.0;
  const int4 n4 = m.nbr4[c];
  const int nr[4] = {n4.x, n4.y, n4.z, n4.w};
  int nb[4];
#pragma unroll
  for (int f = 0; f < 4; f++) nb[f] = (nr[f] >= 0 && nr[f] < NT) ? nr[f] : c;
  double qn[4][4];
#pragma unroll
  for (int f = 0; f < 4; f++) {
    if (Q4) {
      const double4 v = q4[nb[f]];
      qn[f][0] = v.x;
      qn[f][1] = v.y;
      qn[f][2] = v.z;
      qn[f][3] = v.w;
    } else {
#pragma unroll
      for (int k = 0; k < 4; k++) qn[f][k] = prim[k * NT + nb[f]];
    }
  }
#pragma unroll
  for (int k = 0; k < 8; k++) g[k] = 0.0;
  den = 0.0;
#pragma unroll
  for (int f = 0; f < 4; f++) {
    if (f >= nf) break;
    const int idx = f * NP + c;
    const double nxf = m.nx[idx], nyf = m.ny[idx], dlf = m.dl[idx];
    const double wx = nxf * dlf, wy = nyf * dlf;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const double qf = 0.5 * (qc[k] + qn[f][k]);
      g[2 * k] += qf * wx;
      g[2 * k + 1] += qf * wy;
    }
    if (DT) {
      const double vnf = qc[1] * nxf + qc[2] * nyf;
      den += (fabs(vnf) + ac) * dlf;
    }
  }
#pragma unroll
  for (int k = 0; k < 8; k++) g[k] = g[k] * ia;
}

// Gradient records of the face-based forms: the Green-Gauss gradients of (rho, u, v, p) of every
// physical cell, the face value being the mean of the two cell values (a ghost neighbour's value
// carries the boundary state); the states themselves are read from q4.  Work-list entries cover
// record rows NP..NT-1 too (ghost rows), which have nothing to do.
// DT: also del_t of each physical cell (the fused per-cell-dt forms; their Min_dt is formed in
// the last stage's reduction).
// with_bc: first stage of a step; each thread first applies the boundary conditions of its own
// cell's boundary entries (Apply_Boundary_Conditions, as k_bc does), which is exact because a
// ghost row depends only on its owner cell and is read by no other cell's gradient.
template <bool DT>
__global__ void __launch_bounds__(kBlock, 4) k_muscl_gradients(DevMesh m, DevState st, FluxParams fp, BcParams bp,
                                                               int with_bc) {
  pdl_enter();
  const int c = item_index(m.rblk, m.NT);
  const int NP = m.NP, NT = m.NT;
  if (step_done(st.ctl)) return;
  if (c < NP) {
    if (with_bc) {
      const int b0 = m.bptr[c], b1 = m.bptr[c + 1];
      for (int i = b0; i < b1; i++) bc_entry(m, st, bp, m.bidx[i], 0, 0);
    }
    const double4 v = st.q4[c];
    const double qc[4] = {v.x, v.y, v.z, v.w};
    double g[8], den;
    cell_gradients<DT, true>(m, st.prim, st.q4, c, qc, g, den);
    if (st.recf) {
      float4 *r = st.recf + 2 * (size_t)c;
      r[0] = make_float4(float(g[0]), float(g[1]), float(g[2]), float(g[3]));
      r[1] = make_float4(float(g[4]), float(g[5]), float(g[6]), float(g[7]));
    } else {
      double4 *r = reinterpret_cast<double4 *>(st.rec + 8 * (size_t)c);
      r[0] = make_double4(g[0], g[1], g[2], g[3]);
      r[1] = make_double4(g[4], g[5], g[6], g[7]);
    }
    if (DT) st.dtc[c] = cell_dt(m, fp, c, den);
  }
  (void)NT;
}

// ---- Persistent form of one stage for batched solves (no reference counterpart) ----
// One cooperative launch per RK stage does the work of k_muscl_gradients, k_faces and
// k_gather_stage: its resident thread blocks walk the (instance, block) work lists of the active
// instances (record rows, faces, cells), phase after phase, with a grid barrier between the
// phases.  Values written in the same launch by other blocks (records, ghost rows, del_t, face
// fluxes) are read from L2.  Every per-cell and per-face operation is the one the three kernels
// do, so the state is bit-identical to theirs; the error norms of the last stage are reduced over
// the persistent blocks (a different summation order than the three-kernel grid).
//
// The barrier waits are bounded: a block that waits longer than kBarrierCycles (about half a
// second) records CFD_ERR_TIMEOUT in the status word and goes on; once the status is set no block
// waits again, so the launch always ends and the host reads the error.  test_arrivals adds
// arrivals that never come (a test of the timeout path; 0 in every run).
constexpr long long kBarrierCycles = 1ll << 30;
constexpr int kPersistBlock = 128;

__device__ __forceinline__ void grid_barrier(unsigned int *count, unsigned int *gen, int *status,
                                             unsigned int test_arrivals) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int *vgen = gen;
    volatile int *vstatus = status;
    const unsigned int g = *vgen;
    __threadfence();
    const unsigned int arrived = atomicAdd(count, 1u) + 1u;
    if (arrived == gridDim.x + test_arrivals) {
      atomicExch(count, 0u);
      __threadfence();
      atomicAdd(gen, 1u);
    } else {
      const long long t0 = clock64();
      while (*vgen == g) {
        if (*vstatus != 0) break;
        if (clock64() - t0 > kBarrierCycles) {
          atomicCAS(status, 0, 5 /* CFD_ERR_TIMEOUT */);
          break;
        }
        __nanosleep(128);
      }
    }
    __threadfence();
  }
  __syncthreads();
}

// MINB: resident blocks per SM the registers are allocated for (4: 116 registers, no spill; 6: 80
// registers and a small spill, 24 warps per SM; 8: 64 registers).  On a batch of 128 ramps on B200
// the FP64 form runs fastest at 6 (25 % faster than at 4) and the FP32-flux form at 8.
template <typename T, int DISS, int MINB>
__global__ void __launch_bounds__(kPersistBlock, MINB) k_persistent_stage(DevMesh m, DevState st, FluxParams fp,
                                                                       BcParams bp, int kind, int lts, int fuse_final,
                                                                       int keep_delu, int flags, int with_dt,
                                                                       int with_bc, unsigned int test_arrivals) {
  const int NP = m.NP;
  if (step_done(st.ctl)) return;  // every block sees the same flag (written by an earlier launch)
  unsigned int *bar_count = st.counter + 4, *bar_gen = st.counter + 5;
  // Phase 1: gradient records (and del_t), the first stage's boundary conditions.
  // Without work lists (a single solve) the phases walk all rows, faces and cells in chunks.
  const int nr = m.rblk ? m.n_rblk : (NP + kWorkItemBlock - 1) / kWorkItemBlock;
  const int nfb = m.fblk ? m.n_fblk : (m.NF + kWorkFaceBlock - 1) / kWorkFaceBlock;
  const int ncb = m.cblk ? m.n_cblk : (NP + kWorkCellBlock - 1) / kWorkCellBlock;
  for (int w = blockIdx.x; w < nr; w += gridDim.x) {
    const int2 b = m.rblk ? m.rblk[w] : make_int2(w * kWorkItemBlock, min((w + 1) * kWorkItemBlock, NP));
    for (int c = b.x + threadIdx.x; c < b.y; c += blockDim.x) {
      if (c >= NP) continue;
      if (with_bc) {
        const int b0 = m.bptr[c], b1 = m.bptr[c + 1];
        for (int i = b0; i < b1; i++) bc_entry(m, st, bp, m.bidx[i], 0, 0);
      }
      const double4 v = st.q4[c];
      const double qc[4] = {v.x, v.y, v.z, v.w};
      double g[8], den;
      if (with_dt) cell_gradients<true, true>(m, st.prim, st.q4, c, qc, g, den);
      else cell_gradients<false, true>(m, st.prim, st.q4, c, qc, g, den);
      if (st.recf) {
        float4 *r = st.recf + 2 * (size_t)c;
        r[0] = make_float4(float(g[0]), float(g[1]), float(g[2]), float(g[3]));
        r[1] = make_float4(float(g[4]), float(g[5]), float(g[6]), float(g[7]));
      } else {
        double4 *r = reinterpret_cast<double4 *>(st.rec + 8 * (size_t)c);
        r[0] = make_double4(g[0], g[1], g[2], g[3]);
        r[1] = make_double4(g[4], g[5], g[6], g[7]);
      }
      if (with_dt) st.dtc[c] = cell_dt(m, fp, c, den);
    }
  }
  grid_barrier(bar_count, bar_gen, st.status, test_arrivals);
  // Phase 2: face fluxes.
  const int glim = fp.limiter == LIM_REF_MINMOD ? LIM_MINMOD : fp.limiter;
  for (int w = blockIdx.x; w < nfb; w += gridDim.x) {
    const int2 b = m.fblk ? m.fblk[w] : make_int2(w * kWorkFaceBlock, min((w + 1) * kWorkFaceBlock, m.NF));
    for (int i = b.x + threadIdx.x; i < b.y; i += blockDim.x) {
      const int2 on = m.fon[i];
      const int c = on.x, N = on.y;
      const double4 gq = m.fg4[i];
      const T nx = T(gq.x), ny = T(gq.y), dl = T(gq.z), dx = T(gq.w), dy = T(m.fdy[i]);
      const double4 c0 = ldcg4(st.q4 + c), n0 = ldcg4(st.q4 + N);
      const bool nphys = N < NP;
      double4 c1, c2, n1, n2;
      if (sizeof(T) == sizeof(float)) {
        const float4 a = __ldcg(st.recf + 2 * (size_t)c), bb = __ldcg(st.recf + 2 * (size_t)c + 1);
        c1 = make_double4(a.x, a.y, a.z, a.w);
        c2 = make_double4(bb.x, bb.y, bb.z, bb.w);
        if (nphys) {
          const float4 p = __ldcg(st.recf + 2 * (size_t)N), q = __ldcg(st.recf + 2 * (size_t)N + 1);
          n1 = make_double4(p.x, p.y, p.z, p.w);
          n2 = make_double4(q.x, q.y, q.z, q.w);
        } else {
          n1 = c1;
          n2 = c2;
        }
      } else {
        const double4 *rc = reinterpret_cast<const double4 *>(st.rec + 8 * (size_t)c);
        const double4 *rn = reinterpret_cast<const double4 *>(st.rec + 8 * (size_t)N);
        c1 = ldcg4(rc);
        c2 = ldcg4(rc + 1);
        n1 = nphys ? ldcg4(rn) : c1;
        n2 = nphys ? ldcg4(rn + 1) : c2;
      }
      st.F[i] = face_flux_rec<T, DISS>(glim, c0, c1, c2, n0, n1, n2, nx, ny, dl, dx, dy, T(fp.eflin),
                                     T(fp.shock_fix));
    }
  }
  grid_barrier(bar_count, bar_gen, st.status, test_arrivals);
  // Phase 3: gather of each cell's face fluxes in face order and the stage update.
  double dtu = 1e308 * 10.0;
  double e[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int w = blockIdx.x; w < ncb; w += gridDim.x) {
    const int2 b = m.cblk ? m.cblk[w] : make_int2(w * kWorkCellBlock, min((w + 1) * kWorkCellBlock, NP));
    for (int c = b.x + threadIdx.x; c < b.y; c += blockDim.x) {
      double R[4], den = 0.0;
      gather_faces<false, true>(m, st, c, R, den);
      const double dtc = (lts == 1 || first_kind(kind)) ? __ldcg(st.dtc + c) : 0.0;
      const double dt = stage_cell(m, st, bp, c, R, dtc, kind, lts, fuse_final, keep_delu, flags, e);
      dtu = dt < dtu ? dt : dtu;
    }
  }
  if (fuse_final && final_kind(kind)) stage_final_reduce(st, e, dtu);
}

// Patch form of one stage of the face-based per-cell-dt forms: one thread block per patch of up
// to kPatchCells cells does the work of k_muscl_gradients, k_faces and k_gather_stage for its
// cells, with the records and face fluxes in shared memory instead of HBM.
//   1. records (rho, u, v, p and gradients) of its own cells and of its halo cells (the cells
//      across its faces), from the stage's primitives `pin`; del_t of its own cells;
//   2. every face of its own cells (a face to a halo cell is evaluated by both patches, from the
//      owner's side, so both get the same bits), +F into the owner's slot and -F into the
//      neighbour's slot when that cell is its own;
//   3. per own cell: the slots summed in face order and the stage update (stage_cell), which
//      writes the new primitives and the next stage's ghosts to st.prim (a different buffer from
//      `pin`: other blocks are still reading their halo primitives from it).
// Every operation on a value is the one the three-kernel form does, in the same order.
template <int DISS>
__global__ void __launch_bounds__(kPatchCells, 5) k_patch_stage(DevMesh m, DevState st, FluxParams fp, BcParams bp,
                                                                int kind, int lts, int fuse_final, int keep_delu,
                                                                int flags, const double *__restrict__ pin) {
  pdl_enter();
  if (step_done(st.ctl)) return;
  extern __shared__ double smem[];
  const int NP = m.NP, NT = m.NT, rows = m.patch_rows;
  const int b = blockIdx.x, tid = threadIdx.x;
  const int2 pr = m.patch[b];
  const int c0 = pr.x, P = min(pr.y, kPatchCells);
  const int h0 = m.phptr[b], H = m.phptr[b + 1] - h0;
  double *srec = smem;             // [12][rows]: rho, u, v, p, then the 8 gradient terms
  double *sF = smem + 12 * rows;   // [4 slots][4][kPatchCells]
  const int glim = fp.limiter == LIM_REF_MINMOD ? LIM_MINMOD : fp.limiter;

  // The tables are checked on the host; an entry that would still leave its buffer is skipped and
  // reported as a mesh error instead of being used.
  double dtc = 0.0;
  const int nrow = min(P + H, rows);
  for (int l = tid; l < nrow; l += kPatchCells) {
    const int c = l < P ? c0 + l : m.phcell[h0 + l - P];
    if (c < 0 || c >= NP) {
      atomicCAS(&st.status[0], 0, 7 /* CFD_ERR_MESH */);
      continue;
    }
    double qc[4], g[8], den;
#pragma unroll
    for (int k = 0; k < 4; k++) qc[k] = pin[k * NT + c];
    cell_gradients<true>(m, pin, nullptr, c, qc, g, den);
#pragma unroll
    for (int k = 0; k < 4; k++) srec[k * rows + l] = qc[k];
#pragma unroll
    for (int k = 0; k < 8; k++) srec[(4 + k) * rows + l] = g[k];
    if (l < P) {
      dtc = cell_dt(m, fp, c, den);
      st.dtc[c] = dtc;
    }
  }
  __syncthreads();

  const int f0 = m.pfptr[b], f1 = m.pfptr[b + 1];
  for (int j = f0 + tid; j < f1; j += kPatchCells) {
    const PatchFace fe = m.pface[j];
    const int N = fe.N;
    const int lo = fe.rows & 0xFFFF, ln = (int)((unsigned)fe.rows >> 16);
    const int so = fe.slots & 0xFF, sn = (fe.slots >> 8) & 0xFF;
    const bool bad = lo >= nrow || (ln == 0xFFFF ? (N < NP || N >= NT) : ln >= nrow) ||
                     (so != 0xFF && (so > 3 || lo >= P)) || (sn != 0xFF && (sn > 3 || ln >= P));
    if (bad) {
      atomicCAS(&st.status[0], 0, 7 /* CFD_ERR_MESH */);
      continue;
    }
    const double4 c0r = make_double4(srec[lo], srec[rows + lo], srec[2 * rows + lo], srec[3 * rows + lo]);
    const double4 c1r =
        make_double4(srec[4 * rows + lo], srec[5 * rows + lo], srec[6 * rows + lo], srec[7 * rows + lo]);
    const double4 c2r =
        make_double4(srec[8 * rows + lo], srec[9 * rows + lo], srec[10 * rows + lo], srec[11 * rows + lo]);
    double4 n0r, n1r, n2r;
    if (ln == 0xFFFF) {
      // Ghost neighbour: its state, with the owner's gradient.
      n0r = make_double4(pin[N], pin[NT + N], pin[2 * NT + N], pin[3 * NT + N]);
      n1r = c1r;
      n2r = c2r;
    } else {
      n0r = make_double4(srec[ln], srec[rows + ln], srec[2 * rows + ln], srec[3 * rows + ln]);
      n1r = make_double4(srec[4 * rows + ln], srec[5 * rows + ln], srec[6 * rows + ln], srec[7 * rows + ln]);
      n2r = make_double4(srec[8 * rows + ln], srec[9 * rows + ln], srec[10 * rows + ln], srec[11 * rows + ln]);
    }
    const double4 F = face_flux_rec<double, DISS>(glim, c0r, c1r, c2r, n0r, n1r, n2r, fe.nx, fe.ny, fe.dl, fe.dx, fe.dy,
                                                    fp.eflin, fp.shock_fix);
    if (so < 4) {
      sF[(so * 4 + 0) * kPatchCells + lo] = F.x;
      sF[(so * 4 + 1) * kPatchCells + lo] = F.y;
      sF[(so * 4 + 2) * kPatchCells + lo] = F.z;
      sF[(so * 4 + 3) * kPatchCells + lo] = F.w;
    }
    if (sn < 4) {
      sF[(sn * 4 + 0) * kPatchCells + ln] = -F.x;
      sF[(sn * 4 + 1) * kPatchCells + ln] = -F.y;
      sF[(sn * 4 + 2) * kPatchCells + ln] = -F.z;
      sF[(sn * 4 + 3) * kPatchCells + ln] = -F.w;
    }
  }
  __syncthreads();

  double dtu = 1e308 * 10.0;
  double e[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (tid < P && c0 + tid < NP) {
    const int c = c0 + tid;
    const int nf = m.nf[c];
    double R[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int f = 0; f < 4; f++) {
      if (f < nf) {
#pragma unroll
        for (int k = 0; k < 4; k++) R[k] += sF[(f * 4 + k) * kPatchCells + tid];
      }
    }
    // Ghost rows move to the output buffer with their owner (the final stage, and boundary kinds
    // that leave a ghost unchanged, keep its current state); non-final stages overwrite them.
    const int b0 = m.bptr[c], b1 = m.bptr[c + 1];
    for (int q = b0; q < b1; q++) {
      const int g = m.bnd[m.bidx[q]].w;
#pragma unroll
      for (int k = 0; k < 5; k++) st.prim[k * NT + g] = pin[k * NT + g];
      if (st.q4) st.q4[g] = make_double4(pin[g], pin[NT + g], pin[2 * NT + g], pin[3 * NT + g]);
    }
    dtu = stage_cell(m, st, bp, c, R, dtc, kind, lts, fuse_final, keep_delu, flags, e);
  }
  if (fuse_final && final_kind(kind)) stage_final_reduce(st, e, dtu);
}

// ---- Tile form of one stage on a structured block (no reference counterpart) ----
// One thread block per tile of kTileX x kTileY cells does the work of k_muscl_gradients, k_faces
// and k_gather_stage for its cells with everything between them in shared memory:
//   0. the (rho, u, v, p) rows of the tile and of two rings of cells around it (ghost rows
//      beside the block's boundary) from q_in, one coalesced pass per row of the region;
//   1. gradients of the tile's cells and of the halo cells along its four sides (the cells across
//      its boundary faces), del_t of its own cells;
//   2. the flux of every W and S face of its cells, each from its owner's side (a face on the
//      tile boundary is evaluated by both tiles from the same inputs, so both get the same bits);
//   3. per own cell the four fluxes summed in slot order and the stage update (stage_cell), which
//      writes the stage's rows and the next stage's ghost rows to st.q4 (not q_in: other tiles
//      are still reading their halo rows from it).
// Every operation on a value is the one the three-kernel form does, in the same order: the
// gradient terms and the face fluxes are formed per position around the cell and summed in the
// cell's slot order; a slot normal is the owner-side normal negated exactly on the non-owner side
// (checked on the host before the form is offered).
constexpr int kTileX = kTileCellsX;
constexpr int kTileY = kTileCellsY;
constexpr int kTileQW = kTileX + 4, kTileQH = kTileY + 4;  // state region: tile + 2 rings
constexpr int kTileRW = kTileX + 2, kTileRH = kTileY + 2;  // gradient region: tile + 1 ring
constexpr int kTileNW = (kTileX + 1) * kTileY;              // W faces of the tile
constexpr int kTileNS = kTileX * (kTileY + 1);              // S faces of the tile

template <typename T>
struct TileRecT {
  typedef double4 type;
};
template <>
struct TileRecT<float> {
  typedef float4 type;
};

template <typename T>
__host__ __device__ constexpr size_t tile_smem_bytes() {
  return sizeof(double4) * (size_t)(kTileQW * kTileQH + kTileNW + kTileNS) +
         2 * sizeof(typename TileRecT<T>::type) * (size_t)(kTileRW * kTileRH);
}

// acc[k] += t[(R + f) & 3][k] for f = 0..3: position terms summed in the cell's slot order.
template <int R, int K>
__device__ __forceinline__ void rot_sum(const double (&t)[4][K], double (&acc)[K]) {
#pragma unroll
  for (int f = 0; f < 4; f++) {
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] += t[(R + f) & 3][k];
  }
}
template <int K>
__device__ __forceinline__ void slot_order_sum(int r, const double (&t)[4][K], double (&acc)[K]) {
  switch (r) {
    case 0: rot_sum<0, K>(t, acc); break;
    case 1: rot_sum<1, K>(t, acc); break;
    case 2: rot_sum<2, K>(t, acc); break;
    default: rot_sum<3, K>(t, acc); break;
  }
}

// Shared-memory offsets of the four neighbours and the face-table indices of the four faces of
// cell (i, j) at positions E, N, W, S (N and S exchanged when lh).
struct TilePos {
  int dq[4];
  int face[4];  // W-family index (positions 0, 2) or S-family index (1, 3)
};
__device__ __forceinline__ TilePos tile_pos(const TileMesh &tm, int i, int j) {
  TilePos t;
  const int wi = j * (tm.ni + 1) + i, si = j * tm.ni + i;
  t.dq[0] = 1;
  t.dq[2] = -1;
  t.face[0] = wi + 1;
  t.face[2] = wi;
  const int up = tm.lh ? 3 : 1, dn = tm.lh ? 1 : 3;
  t.dq[up] = kTileQW;
  t.dq[dn] = -kTileQW;
  t.face[up] = si + tm.ni;
  t.face[dn] = si;
  return t;
}

// Gradients of physical cell c = (i, j), row qi of the state region, as cell_gradients<DT> forms
// them; with DT also the del_t denominator.
__device__ __forceinline__ void tile_gradients(const DevMesh &m, const DevState &st, const TileMesh &tm,
                                               const double4 *sq, int qi, int c, int i, int j, bool dt, double g[8],
                                               double &den) {
  const unsigned code = tm.code[c];
  const double ia = m.inv_area[c];
  const double ac = dt ? st.prim[4 * m.NT + c] : 0.0;
  const TilePos tp = tile_pos(tm, i, j);
  const double4 qv = sq[qi];
  const double qc[4] = {qv.x, qv.y, qv.z, qv.w};
  double t[4][9];
#pragma unroll
  for (int p = 0; p < 4; p++) {
    const double4 fg = (p & 1) ? tm.fs[tp.face[p]] : tm.fw[tp.face[p]];
    const double4 qn = sq[qi + tp.dq[p]];
    const bool own = (code >> (2 + p)) & 1u;
    const double nxf = own ? fg.x : -fg.x, nyf = own ? fg.y : -fg.y, dlf = fg.z;
    const double wx = nxf * dlf, wy = nyf * dlf;
    const double qnv[4] = {qn.x, qn.y, qn.z, qn.w};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const double qf = 0.5 * (qc[k] + qnv[k]);
      t[p][2 * k] = qf * wx;
      t[p][2 * k + 1] = qf * wy;
    }
    const double vnf = qc[1] * nxf + qc[2] * nyf;
    t[p][8] = (fabs(vnf) + ac) * dlf;
  }
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  slot_order_sum<9>(code & 3u, t, acc);
#pragma unroll
  for (int k = 0; k < 8; k++) g[k] = acc[k] * ia;
  den = acc[8];
}

template <typename T, int DISS>
__global__ void __launch_bounds__(kTileX * kTileY, 2)
    k_tile_stage(DevMesh m, DevState st, FluxParams fp, BcParams bp, TileMesh tm, const double4 *__restrict__ q_in,
                 int kind, int lts, int fuse_final, int keep_delu, int flags, int with_dt) {
  typedef typename TileRecT<T>::type RecV;
  pdl_enter();
  if (step_done(st.ctl)) return;
  extern __shared__ double4 tsm[];
  double4 *sq = tsm;                                           // [QH][QW]
  double4 *sF = sq + kTileQW * kTileQH;                        // W faces [TY][TX + 1], then S faces [TY + 1][TX]
  RecV *srec = reinterpret_cast<RecV *>(sF + kTileNW + kTileNS);  // [RH][RW] x 2
  const int ni = tm.ni, nj = tm.nj, tid = threadIdx.x;
  const int i0 = (blockIdx.x % tm.tiles_i) * kTileX, j0 = (blockIdx.x / tm.tiles_i) * kTileY;
  const int glim = fp.limiter == LIM_REF_MINMOD ? LIM_MINMOD : fp.limiter;

  // 0. States of the region (corners of the outer rings beyond the block are never read).
  for (int t = tid; t < kTileQW * kTileQH; t += blockDim.x) {
    const int jj = t / kTileQW, ii = t - jj * kTileQW;
    const int i = i0 + ii - 2, j = j0 + jj - 2;
    const bool in_i = i >= 0 && i < ni, in_j = j >= 0 && j < nj;
    int r = -1;
    if (in_i && in_j) r = j * ni + i;
    else if (in_j && i == -1) r = tm.gW[j];
    else if (in_j && i == ni) r = tm.gE[j];
    else if (in_i && j == -1) r = tm.gS[i];
    else if (in_i && j == nj) r = tm.gN[i];
    sq[t] = r >= 0 ? q_in[r] : make_double4(0.0, 0.0, 0.0, 0.0);
  }
  __syncthreads();

  // 1. Gradients: own cells (thread tid has cell tid), then the halo strips W, E, S, N.
  double dtc = 0.0;
  constexpr int NG = kTileX * kTileY + 2 * kTileY + 2 * kTileX;
  for (int t = tid; t < NG; t += blockDim.x) {
    int gi, gj;
    if (t < kTileX * kTileY) {
      gi = t % kTileX;
      gj = t / kTileX;
    } else {
      const int u = t - kTileX * kTileY;
      if (u < kTileY) {
        gi = -1;
        gj = u;
      } else if (u < 2 * kTileY) {
        gi = kTileX;
        gj = u - kTileY;
      } else if (u < 2 * kTileY + kTileX) {
        gi = u - 2 * kTileY;
        gj = -1;
      } else {
        gi = u - 2 * kTileY - kTileX;
        gj = kTileY;
      }
    }
    const int i = i0 + gi, j = j0 + gj;
    if (i < 0 || i >= ni || j < 0 || j >= nj) continue;
    const int c = j * ni + i;
    const bool own = t < kTileX * kTileY;
    double g[8], den;
    tile_gradients(m, st, tm, sq, (gj + 2) * kTileQW + gi + 2, c, i, j, own && with_dt, g, den);
    RecV *r = srec + 2 * ((gj + 1) * kTileRW + gi + 1);
    if (sizeof(T) == sizeof(float)) {
      r[0] = RecV{T(float(g[0])), T(float(g[1])), T(float(g[2])), T(float(g[3]))};
      r[1] = RecV{T(float(g[4])), T(float(g[5])), T(float(g[6])), T(float(g[7]))};
    } else {
      r[0] = RecV{T(g[0]), T(g[1]), T(g[2]), T(g[3])};
      r[1] = RecV{T(g[4]), T(g[5]), T(g[6]), T(g[7])};
    }
    if (own && with_dt) {
      dtc = cell_dt(m, fp, c, den);
      st.dtc[c] = dtc;
    }
  }
  __syncthreads();

  // 2. Face fluxes: W faces (i0..i0+TX, rows of the tile), then S faces (columns, j0..j0+TY).
  for (int t = tid; t < kTileNW + kTileNS; t += blockDim.x) {
    int fi, fj, lx, ly, hx, hy, gidx;
    bool lo_phys, hi_phys, ohigh;
    double4 gq;
    double gdy;
    if (t < kTileNW) {
      fj = t / (kTileX + 1);
      fi = t - fj * (kTileX + 1);
      const int i = i0 + fi, j = j0 + fj;
      if (i > ni || j >= nj) continue;
      gidx = j * (ni + 1) + i;
      lx = fi - 1;
      ly = fj;
      hx = fi;
      hy = fj;
      lo_phys = i > 0;
      hi_phys = i < ni;
      gq = tm.fw[gidx];
      gdy = tm.fwdy[gidx];
      ohigh = tm.fwo[gidx] != 0;
    } else {
      const int u = t - kTileNW;
      fj = u / kTileX;
      fi = u - fj * kTileX;
      const int i = i0 + fi, j = j0 + fj;
      if (i >= ni || j > nj) continue;
      gidx = j * ni + i;
      lx = fi;
      ly = fj - 1;
      hx = fi;
      hy = fj;
      lo_phys = j > 0;
      hi_phys = j < nj;
      gq = tm.fs[gidx];
      gdy = tm.fsdy[gidx];
      ohigh = tm.fso[gidx] != 0;
    }
    const int ox = ohigh ? hx : lx, oy = ohigh ? hy : ly, nx_ = ohigh ? lx : hx, ny_ = ohigh ? ly : hy;
    const bool nphys = ohigh ? lo_phys : hi_phys;
    const double4 c0 = sq[(oy + 2) * kTileQW + ox + 2], n0 = sq[(ny_ + 2) * kTileQW + nx_ + 2];
    const RecV *ro = srec + 2 * ((oy + 1) * kTileRW + ox + 1);
    const RecV *rn = nphys ? srec + 2 * ((ny_ + 1) * kTileRW + nx_ + 1) : ro;
    const RecV a = ro[0], b = ro[1], p = rn[0], q = rn[1];
    const double4 c1 = make_double4(a.x, a.y, a.z, a.w), c2 = make_double4(b.x, b.y, b.z, b.w);
    const double4 n1 = make_double4(p.x, p.y, p.z, p.w), n2 = make_double4(q.x, q.y, q.z, q.w);
    sF[t] = face_flux_rec<T, DISS>(glim, c0, c1, c2, n0, n1, n2, T(gq.x), T(gq.y), T(gq.z), T(gq.w), T(gdy),
                                   T(fp.eflin), T(fp.shock_fix));
  }
  __syncthreads();

  // 3. Gather in slot order and stage update of the own cells.
  double dtu = 1e308 * 10.0;
  double e[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  {
    const int tx = tid % kTileX, ty = tid / kTileX;
    const int i = i0 + tx, j = j0 + ty;
    if (i < ni && j < nj) {
      const int c = j * ni + i;
      const unsigned code = tm.code[c];
      const int wE = ty * (kTileX + 1) + tx + 1, wW = wE - 1;
      const int sS = kTileNW + ty * kTileX + tx, sN = sS + kTileX;
      const int pf[4] = {wE, tm.lh ? sS : sN, wW, tm.lh ? sN : sS};
      double t[4][4];
#pragma unroll
      for (int p = 0; p < 4; p++) {
        const double4 F = sF[pf[p]];
        const bool own = (code >> (2 + p)) & 1u;
        t[p][0] = own ? F.x : -F.x;
        t[p][1] = own ? F.y : -F.y;
        t[p][2] = own ? F.z : -F.z;
        t[p][3] = own ? F.w : -F.w;
      }
      double R[4] = {0.0, 0.0, 0.0, 0.0};
      slot_order_sum<4>(code & 3u, t, R);
      // Ghost rows move to the output buffer with their owner (boundary kinds that leave a ghost
      // unchanged, and the final stage, keep its current state); non-final stages overwrite them.
      const int b0 = m.bptr[c], b1 = m.bptr[c + 1];
      for (int q = b0; q < b1; q++) {
        const int g = m.bnd[m.bidx[q]].w;
        st.q4[g] = q_in[g];
      }
      const double dts = (lts == 1 || first_kind(kind)) ? dtc : 0.0;
      dtu = stage_cell(m, st, bp, c, R, dts, kind, lts, fuse_final, keep_delu, flags, e);
    }
  }
  if (fuse_final && final_kind(kind)) stage_final_reduce(st, e, dtu);
}

// ---- TMA form of the tile stage (no reference counterpart) ----
// The work of k_tile_stage, tile by tile and operation by operation the same (so the same bits),
// with every global load moved to the start of the block and made asynchronous:
//   * one thread issues three cp.async.bulk.tensor loads on one mbarrier: the (rho, u, v, p) rows
//     of the tile and two rings (box 36 x 12 of 32-byte rows; rows beyond the block arrive as
//     zeros), and the 48-byte face records of the W faces (35 x 10) and S faces (34 x 11) that the
//     tile's cells and its one-ring halo cells touch;
//   * every thread issues cp.async copies of its own cell's stage inputs (U^n, the stage state,
//     the frozen dt, sound speed and area for del_t) and of the 1/area of the gradient region,
//     and plain loads of the region's slot codes and of the ghost rows beside the block's rim
//     (which the bulk load fills with zeros; they are written after it lands).
// The gradient, face and update phases then read shared memory only.  A face's flux is written
// over the first 32 bytes of its own record (read only by the thread that computes it).
// The mbarrier wait is bounded (kTmaWaitCycles, about half a second): a block whose wait runs out
// records CFD_ERR_TIMEOUT in the status word and ends.
constexpr int kTmaGW = kTileX + 3, kTmaGH = kTileY + 2;  // W-face records: i0-1 .. i0+TX+1, j0-1 .. j0+TY
constexpr int kTmaSW = kTileX + 2, kTmaSH = kTileY + 3;  // S-face records: i0-1 .. i0+TX, j0-1 .. j0+TY+1
constexpr int kTmaRecD = 6;                              // doubles per face record
constexpr int kTmaSin = 11;  // stage inputs per own cell: U^n [4], stage state [4], frozen dt, a, area
// PRE (true): the stage inputs are prefetched into shared memory at block start (96 KB per block,
// 2 blocks per SM); false: they are loaded where they are used, which leaves room for 3 blocks per
// SM (74 KB each, registers capped at 85).
constexpr unsigned kTmaQBytes = kTileQW * kTileQH * 32u;
constexpr unsigned kTmaGWBytes = kTmaGW * kTmaGH * kTmaRecD * 8u;
constexpr unsigned kTmaGSBytes = kTmaSW * kTmaSH * kTmaRecD * 8u;
constexpr long long kTmaWaitCycles = 1ll << 30;
// Threads of the wide variant: 9 warps for the 256 cells of a tile, so the 552 face fluxes take
// two rounds instead of three (the ninth warp has no own cell; it loads and computes gradients and
// faces).  112 registers x 288 threads still leaves two blocks per SM.
constexpr int kTileThreadsWide = 288;

__host__ __device__ constexpr unsigned tma_round128(unsigned x) { return (x + 127u) & ~127u; }

template <typename T, bool PRE>
struct TileTmaLayout {
  static constexpr unsigned q = 0;
  static constexpr unsigned gw = tma_round128(kTmaQBytes);
  static constexpr unsigned gs = gw + tma_round128(kTmaGWBytes);
  static constexpr unsigned rec = gs + tma_round128(kTmaGSBytes);
  static constexpr unsigned sin =
      rec + tma_round128(2u * (unsigned)sizeof(typename TileRecT<T>::type) * kTileRW * kTileRH);
  static constexpr unsigned ia = sin + (PRE ? kTmaSin * kTileX * kTileY * 8u : 0u);
  static constexpr unsigned code = ia + kTileRW * kTileRH * 8u;
  static constexpr unsigned bar = (code + kTileRW * kTileRH + 7u) & ~7u;
  static constexpr unsigned bytes = bar + 8u + 128u;  // + slack to align the base to 128 bytes
};

__device__ __forceinline__ uint32_t sm_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, int x, int y, int z, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sm_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void tma_prefetch_3d(const CUtensorMap *map, int x, int y, int z) {
  asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y), "r"(z)
               : "memory");
}
// L2 prefetch of the bytes [p, p + n) (widened to 16-byte bounds, as the bulk prefetch needs).
__device__ __forceinline__ void l2_prefetch_range(const void *p, size_t n) {
  if (n == 0) return;
  const uintptr_t a = reinterpret_cast<uintptr_t>(p) & ~static_cast<uintptr_t>(15);
  const uintptr_t e = (reinterpret_cast<uintptr_t>(p) + n + 15) & ~static_cast<uintptr_t>(15);
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"(static_cast<unsigned>(e - a)) : "memory");
}
__device__ __forceinline__ bool tma_bar_wait(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > kTmaWaitCycles) return false;
  }
}

// Gradients of cell (gi, gj) of the tile's gradient region (row ri = (gj + 1) * kTileRW + gi + 1)
// as tile_gradients forms them, the face values read from the shared records.
__device__ __forceinline__ void tile_gradients_sm(const TileMesh &tm, const double4 *sq, const double *sgw,
                                                  const double *sgs, int qi, int gi, int gj, unsigned code, double ia,
                                                  double ac, double g[8], double &den) {
  const double *fp4[4];
  const int up = tm.lh ? 3 : 1, dn = tm.lh ? 1 : 3;
  fp4[0] = sgw + kTmaRecD * ((gj + 1) * kTmaGW + gi + 2);
  fp4[2] = sgw + kTmaRecD * ((gj + 1) * kTmaGW + gi + 1);
  fp4[up] = sgs + kTmaRecD * ((gj + 2) * kTmaSW + gi + 1);
  fp4[dn] = sgs + kTmaRecD * ((gj + 1) * kTmaSW + gi + 1);
  int dq[4];
  dq[0] = 1;
  dq[2] = -1;
  dq[up] = kTileQW;
  dq[dn] = -kTileQW;
  const double4 qv = sq[qi];
  const double qc[4] = {qv.x, qv.y, qv.z, qv.w};
  double t[4][9];
#pragma unroll
  for (int p = 0; p < 4; p++) {
    const double2 nxy = *reinterpret_cast<const double2 *>(fp4[p]);
    const double dlf = fp4[p][2];
    const double4 qn = sq[qi + dq[p]];
    const bool own = (code >> (2 + p)) & 1u;
    const double nxf = own ? nxy.x : -nxy.x, nyf = own ? nxy.y : -nxy.y;
    const double wx = nxf * dlf, wy = nyf * dlf;
    const double qnv[4] = {qn.x, qn.y, qn.z, qn.w};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const double qf = 0.5 * (qc[k] + qnv[k]);
      t[p][2 * k] = qf * wx;
      t[p][2 * k + 1] = qf * wy;
    }
    const double vnf = qc[1] * nxf + qc[2] * nyf;
    t[p][8] = (fabs(vnf) + ac) * dlf;
  }
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  slot_order_sum<9>(code & 3u, t, acc);
#pragma unroll
  for (int k = 0; k < 8; k++) g[k] = acc[k] * ia;
  den = acc[8];
}

template <typename T, int DISS, bool PRE, int NTHR>
__global__ void __launch_bounds__(NTHR, PRE ? 2 : 3)
    k_tile_tma(DevMesh m, DevState st, FluxParams fp, BcParams bp, TileMesh tm, const __grid_constant__ TileMaps maps,
               const double4 *__restrict__ q_in, int kind, int lts, int fuse_final, int keep_delu, int flags,
               int with_dt, int ahead) {
  typedef typename TileRecT<T>::type RecV;
  typedef TileTmaLayout<T, PRE> L;
  pdl_enter();
  if (step_done(st.ctl)) return;
  extern __shared__ unsigned char tma_smem_raw[];
  unsigned char *base = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(tma_smem_raw) + 127) &
                                                          ~static_cast<uintptr_t>(127));
  double4 *sq = reinterpret_cast<double4 *>(base + L::q);          // [QH][QW]
  double *sgw = reinterpret_cast<double *>(base + L::gw);          // [GH][GW][6]
  double *sgs = reinterpret_cast<double *>(base + L::gs);          // [SH][SW][6]
  RecV *srec = reinterpret_cast<RecV *>(base + L::rec);            // [RH][RW] x 2
  double *sin = reinterpret_cast<double *>(base + L::sin);         // [kTmaSin][TX * TY]
  double *sia = reinterpret_cast<double *>(base + L::ia);          // [RH][RW]
  unsigned char *scode = base + L::code;                           // [RH][RW]
  const uint32_t bar = sm_u32(base + L::bar);
  const int NP = m.NP, NT = m.NT, ni = tm.ni, nj = tm.nj, tid = threadIdx.x;
  constexpr int NC = kTileX * kTileY;
  static_assert(NTHR >= NC && NTHR % 32 == 0, "one thread per own cell, whole warps");
  static_assert(2 * NTHR >= kTileQW * kTileQH && 2 * NTHR >= kTileRW * kTileRH, "two region rows per thread");
  const int i0 = (blockIdx.x % tm.tiles_i) * kTileX, j0 = (blockIdx.x / tm.tiles_i) * kTileY;
  const int glim = fp.limiter == LIM_REF_MINMOD ? LIM_MINMOD : fp.limiter;
  const bool first = first_kind(kind);
  const bool use_s = kind == 2 || kind == 3 || kind == 22 || kind == 23;

  // 0. Loads.  The mbarrier is initialised, made visible to the async proxy and to the block,
  // then thread 0 posts the byte count and issues the three tensor loads.
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                 "r"(kTmaQBytes + kTmaGWBytes + kTmaGSBytes)
                 : "memory");
    tma_load_3d(sm_u32(sgw), &maps.gw, 0, i0 - 1, j0 - 1, bar);
    tma_load_3d(sm_u32(sgs), &maps.gs, 0, i0 - 1, j0 - 1, bar);
    tma_load_3d(sm_u32(sq), &maps.q, 0, i0 - 2, j0 - 2, bar);
  }
  // Stage inputs of the own cell (thread tid has cell tid of the tile).
  const int tx = tid % kTileX, ty = tid / kTileX;
  const int ci = i0 + tx, cj = j0 + ty;
  const bool own_ok = tid < NC && ci < ni && cj < nj;
  const int c = cj * ni + ci;
  if (PRE && own_ok) {
#pragma unroll
    for (int k = 0; k < 4; k++) cp_async8(sin + k * NC + tid, st.U + (size_t)k * NT + c);
    if (use_s) {
#pragma unroll
      for (int k = 0; k < 4; k++) cp_async8(sin + (4 + k) * NC + tid, st.S + (size_t)k * NP + c);
    }
    if (lts != 1 && !first) cp_async8(sin + 8 * NC + tid, st.dtk + c);
    if (with_dt) {
      cp_async8(sin + 9 * NC + tid, st.prim + 4 * (size_t)NT + c);
      cp_async8(sin + 10 * NC + tid, m.area + c);
    }
  }
  // 1/area and slot codes of the gradient region (tile + one ring, cells inside the block).
  constexpr int NR = kTileRW * kTileRH;
  unsigned char code_r[2] = {0, 0};
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int r = tid + h * NTHR;
    if (r < NR) {
      const int gi = r % kTileRW - 1, gj = r / kTileRW - 1;
      const int i = i0 + gi, j = j0 + gj;
      if (i >= 0 && i < ni && j >= 0 && j < nj) {
        cp_async8(sia + r, m.inv_area + (j * ni + i));
        code_r[h] = tm.code[j * ni + i];
      }
    }
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
  // Ghost rows beside the block's rim in the state region (the tensor load leaves zeros there).
  constexpr int NQ = kTileQW * kTileQH;
  double4 gq[2];
  int gpos[2] = {-1, -1};
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int t = tid + h * NTHR;
    if (t < NQ) {
      const int jj = t / kTileQW, ii = t - jj * kTileQW;
      const int i = i0 + ii - 2, j = j0 + jj - 2;
      const bool in_i = i >= 0 && i < ni, in_j = j >= 0 && j < nj;
      int r = -1;
      if (in_j && i == -1) r = tm.gW[j];
      else if (in_j && i == ni) r = tm.gE[j];
      else if (in_i && j == -1) r = tm.gS[i];
      else if (in_i && j == nj) r = tm.gN[i];
      if (r >= 0) {
        gq[h] = q_in[r];
        gpos[h] = t;
      }
    }
  }
  const bool landed = tma_bar_wait(bar, 0);
  asm volatile("cp.async.wait_all;" ::: "memory");
  if (__syncthreads_or(!landed)) {
    // Record the timeout, then give the copies in flight one more bounded wait before the block
    // (and its shared memory) goes away.
    if (tid == 0) atomicCAS(st.status, 0, 5 /* CFD_ERR_TIMEOUT */);
    tma_bar_wait(bar, 0);
    return;
  }
#pragma unroll
  for (int h = 0; h < 2; h++) {
    if (gpos[h] >= 0) sq[gpos[h]] = gq[h];
    const int r = tid + h * NTHR;
    if (r < NR) scode[r] = code_r[h];
  }
  __syncthreads();
  // Every thread has passed its wait: the mbarrier is retired.
  if (tid == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(bar) : "memory");

  // L2 prefetch of the inputs of tile blockIdx.x + ahead (the tile that starts on this SM's slot in
  // the next wave, ahead = resident blocks of the grid), while this tile computes: its three tensor
  // boxes, and the rows of its stage inputs, 1/area and slot codes.  Hints only; the data are final.
  if (ahead > 0 && blockIdx.x + ahead < gridDim.x) {
    const int nbk = blockIdx.x + ahead;
    const int pi0 = (nbk % tm.tiles_i) * kTileX, pj0 = (nbk / tm.tiles_i) * kTileY;
    if (tid == 0) {
      tma_prefetch_3d(&maps.gw, 0, pi0 - 1, pj0 - 1);
      tma_prefetch_3d(&maps.gs, 0, pi0 - 1, pj0 - 1);
      tma_prefetch_3d(&maps.q, 0, pi0 - 2, pj0 - 2);
    } else if (tid >= 32 && tid < 32 + kTileRH) {
      // rows of the gradient region (1/area, slot codes) and of the own cells (stage inputs)
      const int gj = tid - 32 - 1, j = pj0 + gj;
      if (j >= 0 && j < nj) {
        const int ia0 = max(pi0 - 1, 0), ia1 = min(pi0 + kTileX + 1, ni);
        const size_t r0 = (size_t)j * ni;
        l2_prefetch_range(m.inv_area + r0 + ia0, (size_t)(ia1 - ia0) * 8);
        l2_prefetch_range(tm.code + r0 + ia0, (size_t)(ia1 - ia0));
        if (PRE && gj >= 0 && gj < kTileY) {
          const int o1 = min(pi0 + kTileX, ni);
          const size_t nb8 = (size_t)(o1 - pi0) * 8;
#pragma unroll
          for (int k = 0; k < 4; k++) l2_prefetch_range(st.U + (size_t)k * NT + r0 + pi0, nb8);
          if (use_s) {
#pragma unroll
            for (int k = 0; k < 4; k++) l2_prefetch_range(st.S + (size_t)k * NP + r0 + pi0, nb8);
          }
          if (lts != 1 && !first) l2_prefetch_range(st.dtk + r0 + pi0, nb8);
          if (with_dt) {
            l2_prefetch_range(st.prim + 4 * (size_t)NT + r0 + pi0, nb8);
            l2_prefetch_range(m.area + r0 + pi0, nb8);
          }
        }
      }
    }
  }

  // 1. Gradients: own cells (thread tid has cell tid), then the halo strips W, E, S, N.
  double dtc = 0.0;
  constexpr int NG = kTileX * kTileY + 2 * kTileY + 2 * kTileX;
  for (int t = tid; t < NG; t += blockDim.x) {
    int gi, gj;
    if (t < kTileX * kTileY) {
      gi = t % kTileX;
      gj = t / kTileX;
    } else {
      const int u = t - kTileX * kTileY;
      if (u < kTileY) {
        gi = -1;
        gj = u;
      } else if (u < 2 * kTileY) {
        gi = kTileX;
        gj = u - kTileY;
      } else if (u < 2 * kTileY + kTileX) {
        gi = u - 2 * kTileY;
        gj = -1;
      } else {
        gi = u - 2 * kTileY - kTileX;
        gj = kTileY;
      }
    }
    const int i = i0 + gi, j = j0 + gj;
    if (i < 0 || i >= ni || j < 0 || j >= nj) continue;
    const bool own = t < kTileX * kTileY;
    const bool dt = own && with_dt;
    const int ri = (gj + 1) * kTileRW + gi + 1;
    double g[8], den;
    const double ac = dt ? (PRE ? sin[9 * NC + t] : st.prim[4 * (size_t)NT + c]) : 0.0;
    tile_gradients_sm(tm, sq, sgw, sgs, (gj + 2) * kTileQW + gi + 2, gi, gj, scode[ri], sia[ri], ac, g, den);
    RecV *r = srec + 2 * ri;
    if (sizeof(T) == sizeof(float)) {
      r[0] = RecV{T(float(g[0])), T(float(g[1])), T(float(g[2])), T(float(g[3]))};
      r[1] = RecV{T(float(g[4])), T(float(g[5])), T(float(g[6])), T(float(g[7]))};
    } else {
      r[0] = RecV{T(g[0]), T(g[1]), T(g[2]), T(g[3])};
      r[1] = RecV{T(g[4]), T(g[5]), T(g[6]), T(g[7])};
    }
    if (dt) {
      dtc = cell_dt_a(fp, PRE ? sin[10 * NC + t] : m.area[c], den);
      st.dtc[c] = dtc;
    }
  }
  __syncthreads();

  // 2. Face fluxes: W faces (i0..i0+TX, rows of the tile), then S faces (columns, j0..j0+TY);
  // each flux over the first four doubles of its own record.
  for (int t = tid; t < kTileNW + kTileNS; t += blockDim.x) {
    int lx, ly, hx, hy;
    bool lo_phys, hi_phys;
    double *rec;
    if (t < kTileNW) {
      const int fj = t / (kTileX + 1), fi = t - fj * (kTileX + 1);
      const int i = i0 + fi, j = j0 + fj;
      if (i > ni || j >= nj) continue;
      rec = sgw + kTmaRecD * ((fj + 1) * kTmaGW + fi + 1);
      lx = fi - 1;
      ly = fj;
      hx = fi;
      hy = fj;
      lo_phys = i > 0;
      hi_phys = i < ni;
    } else {
      const int u = t - kTileNW;
      const int fj = u / kTileX, fi = u - fj * kTileX;
      const int i = i0 + fi, j = j0 + fj;
      if (i >= ni || j > nj) continue;
      rec = sgs + kTmaRecD * ((fj + 1) * kTmaSW + fi + 1);
      lx = fi;
      ly = fj - 1;
      hx = fi;
      hy = fj;
      lo_phys = j > 0;
      hi_phys = j < nj;
    }
    const double2 g01 = *reinterpret_cast<const double2 *>(rec);
    const double2 g23 = *reinterpret_cast<const double2 *>(rec + 2);
    const double2 g45 = *reinterpret_cast<const double2 *>(rec + 4);
    const bool ohigh = g45.y != 0.0;
    const int ox = ohigh ? hx : lx, oy = ohigh ? hy : ly, nx_ = ohigh ? lx : hx, ny_ = ohigh ? ly : hy;
    const bool nphys = ohigh ? lo_phys : hi_phys;
    const double4 c0 = sq[(oy + 2) * kTileQW + ox + 2], n0 = sq[(ny_ + 2) * kTileQW + nx_ + 2];
    const RecV *ro = srec + 2 * ((oy + 1) * kTileRW + ox + 1);
    const RecV *rn = nphys ? srec + 2 * ((ny_ + 1) * kTileRW + nx_ + 1) : ro;
    const RecV a = ro[0], b = ro[1], p = rn[0], q = rn[1];
    const double4 c1 = make_double4(a.x, a.y, a.z, a.w), c2 = make_double4(b.x, b.y, b.z, b.w);
    const double4 n1 = make_double4(p.x, p.y, p.z, p.w), n2 = make_double4(q.x, q.y, q.z, q.w);
    const double4 F = face_flux_rec<T, DISS>(glim, c0, c1, c2, n0, n1, n2, T(g01.x), T(g01.y), T(g23.x), T(g23.y),
                                             T(g45.x), T(fp.eflin), T(fp.shock_fix));
    *reinterpret_cast<double2 *>(rec) = make_double2(F.x, F.y);
    *reinterpret_cast<double2 *>(rec + 2) = make_double2(F.z, F.w);
  }
  __syncthreads();

  // 3. Gather in slot order and stage update of the own cells.
  double dtu = 1e308 * 10.0;
  double e[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (own_ok) {
    const unsigned code = scode[(ty + 1) * kTileRW + tx + 1];
    const double *fE = sgw + kTmaRecD * ((ty + 1) * kTmaGW + tx + 2);
    const double *fW = sgw + kTmaRecD * ((ty + 1) * kTmaGW + tx + 1);
    const double *fN = sgs + kTmaRecD * ((ty + 2) * kTmaSW + tx + 1);
    const double *fS = sgs + kTmaRecD * ((ty + 1) * kTmaSW + tx + 1);
    const double *pf[4] = {fE, tm.lh ? fS : fN, fW, tm.lh ? fN : fS};
    double t[4][4];
#pragma unroll
    for (int p = 0; p < 4; p++) {
      const double2 a = *reinterpret_cast<const double2 *>(pf[p]);
      const double2 b = *reinterpret_cast<const double2 *>(pf[p] + 2);
      const bool own = (code >> (2 + p)) & 1u;
      t[p][0] = own ? a.x : -a.x;
      t[p][1] = own ? a.y : -a.y;
      t[p][2] = own ? b.x : -b.x;
      t[p][3] = own ? b.y : -b.y;
    }
    double R[4] = {0.0, 0.0, 0.0, 0.0};
    slot_order_sum<4>(code & 3u, t, R);
    // Ghost rows move to the output buffer with their owner (as in k_tile_stage).
    const int b0 = m.bptr[c], b1 = m.bptr[c + 1];
    for (int q = b0; q < b1; q++) {
      const int g = m.bnd[m.bidx[q]].w;
      st.q4[g] = q_in[g];
    }
    const double dts = (lts == 1 || first) ? dtc : 0.0;
    if (PRE) {
      StageIn in;
      in.invA = sia[(ty + 1) * kTileRW + tx + 1];
#pragma unroll
      for (int k = 0; k < 4; k++) in.Un[k] = sin[k * NC + tid];
      if (use_s) {
#pragma unroll
        for (int k = 0; k < 4; k++) in.Sk[k] = sin[(4 + k) * NC + tid];
      }
      const double dt_frozen = (lts != 1 && !first) ? sin[8 * NC + tid] : 0.0;
      dtu = stage_cell_in(m, st, bp, c, R, dts, dt_frozen, in, kind, lts, fuse_final, keep_delu, flags, e);
    } else {
      dtu = stage_cell(m, st, bp, c, R, dts, kind, lts, fuse_final, keep_delu, flags, e);
    }
  }
  // The state region is no longer read: its first 2.4 KB hold the reduction scratch.
  if (fuse_final && final_kind(kind)) stage_final_reduce_sm(st, e, dtu, reinterpret_cast<double *>(sq));
}

__global__ void k_gradient(DevMesh m, DevState st, int var, double *grad) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.NP) return;
  double g0, g1;
  gg_gradient(m, st.prim + (size_t)var * m.NT, c, g0, g1);
  grad[2 * c] = g0;
  grad[2 * c + 1] = g1;
}

// Compute_Gradient_Refinement_Indicator (src/Grid_Refine_Functions.cpp:8-31).
__global__ void k_amr_indicator(DevMesh m, DevState st, double *ind) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.NP) return;
  double v = 0.0;
  const double h = sqrt(m.area[c]);
  double g0, g1;
  gg_gradient(m, st.prim, c, g0, g1);
  v += sqrt(g0 * g0 + g1 * g1) * h;
  gg_gradient(m, st.prim + 3 * (size_t)m.NT, c, g0, g1);
  const double P = st.prim[3 * m.NT + c];
  if (P > 1e-14) v += (sqrt(g0 * g0 + g1 * g1) / P) * h;
  ind[c] = v;
}

__global__ void k_set_ctl(double *ctl, int idx, double v) { ctl[idx] = v; }

// sum(R_rho^2) over one instance's cell range per block: fixed per-thread strides and a fixed
// block tree, so the value is deterministic.
__global__ void k_instance_residual(const double *R, const int *start, const int *end, double *out) {
  __shared__ double sh[32];
  const int i = blockIdx.x;
  double acc = 0.0;
  for (int c = start[i] + threadIdx.x; c < end[i]; c += blockDim.x) acc += R[c] * R[c];
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) out[i] = acc;
}

// ---- Pointwise evaluation of the face functions (checkers' entry points) ----
// phi(a, b) of the limiter family for n pairs.
__global__ void k_eval_limiter(int limiter, const double *a, const double *b, int n, double *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = phi_ab<double>(limiter, a[i], b[i]);
}

// Face flux of scheme `scheme` (3 Roe average + dissipation, 6 AUSM, 7 HLLC, 8 reference GPU AUSM)
// for n conserved left/right states [n][4], outward normals [n][2] and lengths [n]; T is the
// arithmetic precision (the states are rounded to T first, as in the FP32-flux form).  Primitive
// variables for Roe and HLLC come from the reference EOS (eos_prim).
template <typename T>
__global__ void k_eval_face_flux(int scheme, const double *UL, const double *UR, const double *nrm, const double *len,
                                 int n, double *F) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const T nx = T(nrm[2 * i]), ny = T(nrm[2 * i + 1]), dl = T(len[i]);
  T A[4], D[4] = {T(0.0), T(0.0), T(0.0), T(0.0)};
  const T uL[4] = {T(UL[4 * i]), T(UL[4 * i + 1]), T(UL[4 * i + 2]), T(UL[4 * i + 3])};
  const T uR[4] = {T(UR[4 * i]), T(UR[4 * i + 1]), T(UR[4 * i + 2]), T(UR[4 * i + 3])};
  if (scheme == 6) {
    ausm_face<T>(uL, uR, nx, ny, dl, A);
  } else if (scheme == 8) {
    ausm_gpu_face<T>(uL, uR, nx, ny, dl, A);
  } else {
    Prim pl, pr;
    eos_prim(UL[4 * i], UL[4 * i + 1], UL[4 * i + 2], UL[4 * i + 3], pl);
    eos_prim(UR[4 * i], UR[4 * i + 1], UR[4 * i + 2], UR[4 * i + 3], pr);
    const T qL[5] = {T(pl.rho), T(pl.u), T(pl.v), T(pl.p), T(pl.a)};
    const T qR[5] = {T(pr.rho), T(pr.u), T(pr.v), T(pr.p), T(pr.a)};
    if (scheme == 7) {
      hllc_face<T>(qL, uL, qR, uR, nx, ny, dl, A);
    } else {
      average_flux<T>(qL[0], qL[1], qL[2], qL[3], qR[0], qR[1], qR[2], qR[3], nx, ny, dl, A);
      roe_1o<T>(qL[0], qL[1], qL[2], qL[3], qL[4], qR[0], qR[1], qR[2], qR[3], qR[4], nx, ny, dl, false, D);
    }
  }
#pragma unroll
  for (int k = 0; k < 4; k++) F[4 * i + k] = double(A[k] - D[k]);
}

// ---- AMR tagging (TagRefinableCells, src/Grid_Refine_Functions.cpp:33-63) on the device ----
// Top-fraction rule: the nRefine largest indicators are found by a radix select over the bit
// patterns of the (non-negative) indicators, 8 bits per pass; ties at the cut are resolved by a
// second radix select over the reference cell ids (lowest ids first).  Counts are integer
// atomics, so the result is deterministic.
struct SelectState {
  unsigned long long prefix;  // key digits fixed so far
  unsigned long long mask;    // bits of prefix that are fixed
  long long remaining;        // rank still to find inside the current prefix
  long long above;            // number of keys strictly beyond the prefix
};

__device__ __forceinline__ unsigned long long amr_key(double v) {
  return v > 0.0 ? static_cast<unsigned long long>(__double_as_longlong(v)) : 0ull;
}

// Histogram of the next 8-bit digit of keys inside the current prefix.  mode 0: keys are the
// indicator bits (descending select); mode 1: keys are reference ids among cells whose indicator
// key equals `match` (ascending select).
__global__ void k_amr_hist(const double *ind, const int *ref, int NP, const SelectState *sel, int shift, int mode,
                           unsigned long long match, unsigned int *hist) {
  __shared__ unsigned int h[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0u;
  __syncthreads();
  const unsigned long long prefix = sel->prefix, mask = sel->mask;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < NP; c += gridDim.x * blockDim.x) {
    unsigned long long key;
    if (mode == 0) key = amr_key(ind[c]);
    else {
      if (amr_key(ind[c]) != match) continue;
      key = static_cast<unsigned long long>(ref[c]);
    }
    if ((key & mask) == prefix) atomicAdd(&h[(key >> shift) & 255ull], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 256; i += blockDim.x)
    if (h[i]) atomicAdd(&hist[i], h[i]);
}

// Picks the digit holding the wanted rank (from the top for mode 0, from the bottom for mode 1)
// and clears the histogram for the next pass.
__global__ void k_amr_pick(SelectState *sel, int shift, int mode, unsigned int *hist) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  long long rem = sel->remaining;
  long long skipped = 0;
  int digit = 0;
  for (int i = 0; i < 256; i++) {
    const int d = mode == 0 ? 255 - i : i;
    const long long cnt = hist[d];
    if (rem <= cnt) {
      digit = d;
      break;
    }
    rem -= cnt;
    skipped += cnt;
  }
  sel->prefix |= static_cast<unsigned long long>(digit) << shift;
  sel->mask |= 255ull << shift;
  sel->remaining = rem;
  sel->above += skipped;
  for (int i = 0; i < 256; i++) hist[i] = 0u;
}

__global__ void k_amr_tag(const double *ind, const int *ref, int NP, double threshold, int top, const SelectState *sel,
                          const SelectState *sel_ref, uint8_t *tags) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= NP) return;
  const double v = ind[c];
  bool t;
  if (!top) {
    t = v > threshold;
  } else {
    const unsigned long long k = amr_key(v), K = sel->prefix;
    const bool in = k > K || (k == K && static_cast<unsigned long long>(ref[c]) <= sel_ref->prefix);
    t = in && v >= threshold;
  }
  tags[c] = t ? 1 : 0;
}

// Reference-order AoS rows [NT][4] <-> device-order SoA planes [4][NT] (perm: device -> reference).
__global__ void k_import_aos(const double *__restrict__ aos, const int *__restrict__ perm, int NP, int NT, double *U) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NT) return;
  const int r = i < NP ? perm[i] : i;
  const double4 v = reinterpret_cast<const double4 *>(aos)[r];
  U[i] = v.x;
  U[NT + i] = v.y;
  U[2 * NT + i] = v.z;
  U[3 * NT + i] = v.w;
}

__global__ void k_export_aos(const double *__restrict__ U, const int *__restrict__ perm, int NP, int NT, int ld,
                             double *aos) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NT) return;
  const int r = i < NP ? perm[i] : i;
  reinterpret_cast<double4 *>(aos)[r] = make_double4(U[i], U[ld + i], U[2 * ld + i], U[3 * ld + i]);
}

inline int nblk(int n, int b) { return (n + b - 1) / b; }

}  // namespace

// Upper bound on the thread blocks of any flux-kernel variant (sizes the partial-min buffer).
int flux_block_count(int NP) {
  int a = nblk(NP, kFluxBlock), b = nblk(4 * NP, kFlux4Block), c = nblk(NP, kBlock);
  return a > b ? (a > c ? a : c) : (b > c ? b : c);
}

int launch_prim_all(cudaStream_t s, const DevMesh &m, DevState &st) {
  k_prim_all<<<nblk(m.NT, kBlock), kBlock, 0, s>>>(m, st);
  return 1;
}

int launch_bc(cudaStream_t s, const DevMesh &m, DevState &st, const BcParams &bp, int src_is_S, int cur_is_S) {
  if (m.NB == 0) return 0;
  if (m.bblk) {
    if (m.n_bblk == 0) return 0;
    launch_k(m, k_bc, m.n_bblk, kWorkItemBlock, s, m, st, bp, src_is_S, cur_is_S);
  } else {
    launch_k(m, k_bc, nblk(m.NB, kBlock), kBlock, s, m, st, bp, src_is_S, cur_is_S);
  }
  return 1;
}

int launch_instance_residual(cudaStream_t s, const DevState &st, int NP, const int *start, const int *end, int n,
                             double *out) {
  (void)NP;
  if (n <= 0) return 0;
  k_instance_residual<<<n, 256, 0, s>>>(st.R, start, end, out);
  return 1;
}

template <typename T>
void launch_faces_t(cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp);

// Lax_Fedrichs (src/Numerical_Method.cpp:459-481): U_c = 0.25 (U_N0 + U_N1 + U_N2 + U_N3) -
// Min_dt A^-1 R_c, in place.  The reference sweeps the cells in its own order, so a cell reads the
// neighbours that come before it with their new values and the others with their old ones.  One
// launch per wavefront level: a cell's level is one more than the highest level of its earlier
// neighbours, so no two cells of a level are neighbours, a level's earlier neighbours are all
// done and its later ones not yet started; every cell then sees what the sequential sweep shows
// it, and the sums are the same bits.
__global__ void __launch_bounds__(kBlock) k_lax_friedrichs(DevMesh m, DevState st, const int *cells, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = cells[i];
  const int NP = m.NP, NT = m.NT;
  const int n0 = m.nbr[c], n1 = m.nbr[NP + c], n2 = m.nbr[2 * NP + c], n3 = m.nbr[3 * NP + c];
  const double Dt = st.ctl[CTL_DTMIN];
  const double ia = m.inv_area[c];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const double *U = st.U + (size_t)k * NT;
    st.U[(size_t)k * NT + c] = 0.25 * (U[n0] + U[n1] + U[n2] + U[n3]) - Dt * ia * st.R[(size_t)k * NP + c];
  }
}

int launch_lax_friedrichs(cudaStream_t s, const DevMesh &m, DevState &st, const int *cells,
                          const std::vector<int> &level_start) {
  int n = 0;
  for (size_t l = 0; l + 1 < level_start.size(); l++) {
    const int b = level_start[l], e = level_start[l + 1];
    k_lax_friedrichs<<<nblk(e - b, kBlock), kBlock, 0, s>>>(m, st, cells + b, e - b);
    n++;
  }
  return n;
}

// A per-cell form that reads conserved states (limiter, LLF, MOVERS, MOVERS_NWSC, AUSM, HLLC): the
// build that reads them from U alone when no stage state can be asked for (the reference's
// integrators, and the first stage of every form), else the one that picks U or the stage state
// per cell.  Same bits either way.
template <int DISS, int ORDER>
void launch_flux_src(int g, cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp, int src_is_S) {
  if (fp.consistent && src_is_S) k_flux<DISS, ORDER, 1, true><<<g, kFluxBlock, 0, s>>>(m, st, fp, src_is_S);
  else k_flux<DISS, ORDER, 1, false><<<g, kFluxBlock, 0, s>>>(m, st, fp, src_is_S);
}

// The second-order per-cell forms with the directional limiter (ROE_2O, RICCA_2O, MOVERS_NWSC_2O):
// one build per register budget (minimum resident blocks of 128 threads per SM: 1 unconstrained,
// 6 or 8), chosen by fp.flux_minb; every build gives the same bits.
template <int DISS>
void launch_flux_limited(int g, cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp, int src_is_S) {
  if (!(fp.consistent && src_is_S)) {
    switch (fp.flux_minb) {
      case 6: k_flux<DISS, 2, 6, false><<<g, kFluxBlock, 0, s>>>(m, st, fp, src_is_S); break;
      case 8: k_flux<DISS, 2, 8, false><<<g, kFluxBlock, 0, s>>>(m, st, fp, src_is_S); break;
      default: k_flux<DISS, 2, 1, false><<<g, kFluxBlock, 0, s>>>(m, st, fp, src_is_S); break;
    }
    return;
  }
  switch (fp.flux_minb) {
    case 6: k_flux<DISS, 2, 6><<<g, kFluxBlock, 0, s>>>(m, st, fp, src_is_S); break;
    case 8: k_flux<DISS, 2, 8><<<g, kFluxBlock, 0, s>>>(m, st, fp, src_is_S); break;
    default: k_flux<DISS, 2><<<g, kFluxBlock, 0, s>>>(m, st, fp, src_is_S); break;
  }
}

int launch_flux(cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp, int src_is_S) {
  int n = 0;
  if (fp.second_order && fp.muscl) n += launch_muscl_gradients(s, m, st, fp, 0);
  if (fp.second_order && fp.muscl && m.NF > 0) {
    if (fp.precision == 1) launch_faces_t<float>(s, m, st, fp);
    else launch_faces_t<double>(s, m, st, fp);
    k_gather<<<nblk(m.NP, kFluxBlock), kFluxBlock, 0, s>>>(m, st, fp);
    return n + 2;
  }
  if (fp.weno) {
    k_weno<<<nblk(m.NP, kFluxBlock), kFluxBlock, 0, s>>>(m, st, fp, src_is_S);
    return n + 1;
  }
  if (fp.lanes == 1) {
    const int g = nblk(m.NP, kFluxBlock);
    if (fp.dissipation == 3 && !fp.second_order) k_flux<3, 1><<<g, kFluxBlock, 0, s>>>(m, st, fp, src_is_S);
    else if (fp.dissipation == 2 && !fp.second_order) launch_flux_src<2, 1>(g, s, m, st, fp, src_is_S);
    else if (fp.dissipation == 2) launch_flux_src<2, 2>(g, s, m, st, fp, src_is_S);
    else if (fp.dissipation == 4 && !fp.second_order) k_flux<4, 1><<<g, kFluxBlock, 0, s>>>(m, st, fp, src_is_S);
    else if (fp.dissipation == 5 && !fp.second_order) launch_flux_src<5, 1>(g, s, m, st, fp, src_is_S);
    else if (fp.dissipation == 6) launch_flux_src<6, 1>(g, s, m, st, fp, src_is_S);
    else if (fp.dissipation == 7) launch_flux_src<7, 1>(g, s, m, st, fp, src_is_S);
    else if (fp.dissipation == 3) launch_flux_limited<3>(g, s, m, st, fp, src_is_S);
    else if (fp.dissipation == 4) launch_flux_limited<4>(g, s, m, st, fp, src_is_S);
    else if (fp.dissipation == 5) launch_flux_limited<5>(g, s, m, st, fp, src_is_S);
    else launch_flux_src<1, 1>(g, s, m, st, fp, src_is_S);
  } else {
    const int g = nblk(4 * m.NP, kFlux4Block);
    if (fp.dissipation == 3 && !fp.second_order) k_flux4<3, 1><<<g, kFlux4Block, 0, s>>>(m, st, fp, src_is_S);
    else if (fp.dissipation == 2 && !fp.second_order) k_flux4<2, 1><<<g, kFlux4Block, 0, s>>>(m, st, fp, src_is_S);
    else if (fp.dissipation == 2) k_flux4<2, 2><<<g, kFlux4Block, 0, s>>>(m, st, fp, src_is_S);
    else if (fp.dissipation == 4 && !fp.second_order) k_flux4<4, 1><<<g, kFlux4Block, 0, s>>>(m, st, fp, src_is_S);
    else if (fp.dissipation == 4) k_flux4<4, 2><<<g, kFlux4Block, 0, s>>>(m, st, fp, src_is_S);
    else if (fp.dissipation == 5 && !fp.second_order) k_flux4<5, 1><<<g, kFlux4Block, 0, s>>>(m, st, fp, src_is_S);
    else if (fp.dissipation == 5) k_flux4<5, 2><<<g, kFlux4Block, 0, s>>>(m, st, fp, src_is_S);
    else if (fp.dissipation == 6) k_flux4<6, 1><<<g, kFlux4Block, 0, s>>>(m, st, fp, src_is_S);
    else if (fp.dissipation == 7) k_flux4<7, 1><<<g, kFlux4Block, 0, s>>>(m, st, fp, src_is_S);
    else if (fp.dissipation == 3) k_flux4<3, 2><<<g, kFlux4Block, 0, s>>>(m, st, fp, src_is_S);
    else k_flux4<1, 1><<<g, kFlux4Block, 0, s>>>(m, st, fp, src_is_S);
  }
  return n + 1;
}

int launch_stage(cudaStream_t s, const DevMesh &m, DevState &st, int kind, int lts, int fuse_final, int keep_delu) {
  if (m.cblk) k_stage<<<m.n_cblk, kWorkCellBlock, 0, s>>>(m, st, kind, lts, fuse_final, keep_delu);
  else k_stage<<<nblk(m.NP, kBlock), kBlock, 0, s>>>(m, st, kind, lts, fuse_final, keep_delu);
  return 1;
}

int launch_gather(cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp) {
  const int g = m.cblk ? m.n_cblk : nblk(m.NP, kFluxBlock);
  k_gather<<<g, kFluxBlock, 0, s>>>(m, st, fp);
  return 1;
}

// Flux scheme of the face kernels: 3 (Roe) becomes 103 when the Roe options are on.
__host__ __forceinline__ int face_scheme(const FluxParams &fp) {
  return fp.dissipation == 3 && (fp.eflin > 0.0 || fp.shock_fix > 0.0) ? 103 : fp.dissipation;
}

template <typename T, int MINB>
void launch_faces_b(cudaStream_t s, int g, int b, const DevMesh &m, DevState &st, const FluxParams &fp) {
  if (face_scheme(fp) == 103) launch_k(m, k_faces<T, 103, MINB>, g, b, s, m, st, fp);
  else if (fp.dissipation == 6) launch_k(m, k_faces<T, 6, MINB>, g, b, s, m, st, fp);
  else if (fp.dissipation == 7) launch_k(m, k_faces<T, 7, MINB>, g, b, s, m, st, fp);
  else if (fp.dissipation == 8) launch_k(m, k_faces<T, 8, MINB>, g, b, s, m, st, fp);
  else launch_k(m, k_faces<T, 3, MINB>, g, b, s, m, st, fp);
}

// Launch shapes of the face kernel (identical results).  The double Roe kernel needs 86
// registers: 256-thread blocks then fit 2 per SM (16 warps, shape 0), 256-thread blocks capped
// at 80 registers fit 3 (24 warps, a few bytes of spill; shape 1), 128-thread blocks fit 5 (20
// warps; shape 2), 128-thread blocks capped at 72 or 64 registers fit 7 or 8 (28 or 32 warps,
// 44 or 88 bytes of spill held in L1; shapes 3 and 4).  Work lists hold kWorkFaceBlock (128)
// faces per block, so with them every shape runs 128-thread blocks.
template <typename T>
void launch_faces_t(cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp) {
  const bool wl = m.fblk != nullptr;
  const int g128 = wl ? m.n_fblk : nblk(m.NF, 128);
  const int g = wl ? m.n_fblk : nblk(m.NF, 256), b = wl ? 128 : 256;
  if (fp.faces_shape == 4) launch_faces_b<T, 8>(s, g128, 128, m, st, fp);
  else if (fp.faces_shape == 3) launch_faces_b<T, 7>(s, g128, 128, m, st, fp);
  else if (fp.faces_shape == 2) launch_faces_b<T, 1>(s, g128, 128, m, st, fp);
  else if (fp.faces_shape == 1) launch_faces_b<T, 3>(s, g, b, m, st, fp);
  else launch_faces_b<T, 1>(s, g, b, m, st, fp);
}

int launch_faces(cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp) {
  if (m.fblk && m.n_fblk == 0) return 0;
  if (fp.precision == 1) launch_faces_t<float>(s, m, st, fp);
  else launch_faces_t<double>(s, m, st, fp);
  return 1;
}

int gather_stage_wave_blocks() {
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gather_stage<true>, kFluxBlock, 0) != cudaSuccess)
    return 0;
  return sms * per_sm;
}

int launch_gather_stage(cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp, const BcParams &bp,
                        int kind, int lts, int fuse_final, int keep_delu, int flags) {
  const int g = m.cblk ? m.n_cblk : nblk(m.NP, kFluxBlock);
  if (!m.cblk && fuse_final && final_kind(kind) && m.wave_blocks > 0 && g > m.wave_blocks)
    launch_k(m, k_gather_stage<true>, m.wave_blocks, kFluxBlock, s, m, st, fp, bp, kind, lts, fuse_final, keep_delu,
             flags);
  else
    launch_k(m, k_gather_stage<false>, g, kFluxBlock, s, m, st, fp, bp, kind, lts, fuse_final, keep_delu, flags);
  return 1;
}

template <typename T>
int tile_prepare_t() {
  const int n = static_cast<int>(tile_smem_bytes<T>());
  return cudaFuncSetAttribute(k_tile_stage<T, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, n) == cudaSuccess &&
         cudaFuncSetAttribute(k_tile_stage<T, 103>, cudaFuncAttributeMaxDynamicSharedMemorySize, n) == cudaSuccess &&
         cudaFuncSetAttribute(k_tile_stage<T, 6>, cudaFuncAttributeMaxDynamicSharedMemorySize, n) == cudaSuccess &&
         cudaFuncSetAttribute(k_tile_stage<T, 7>, cudaFuncAttributeMaxDynamicSharedMemorySize, n) == cudaSuccess &&
         cudaFuncSetAttribute(k_tile_stage<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, n) == cudaSuccess;
}

int tile_prepare() {
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
  if (tile_smem_bytes<double>() > (size_t)optin) return 0;
  const int ok = tile_prepare_t<double>() && tile_prepare_t<float>();
  cudaGetLastError();
  return ok;
}

template <typename T>
void launch_tile_t(cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp, const BcParams &bp,
                   const TileMesh &tm, const double4 *q_in, int kind, int lts, int fin, int keep_delu, int flags,
                   int with_dt) {
  const unsigned g = static_cast<unsigned>(tm.tiles_i) * static_cast<unsigned>(tm.tiles_j);
  const unsigned b = kTileX * kTileY;
  const size_t sm = tile_smem_bytes<T>();
  const int sch = face_scheme(fp);
  if (sch == 103)
    launch_ks(m, k_tile_stage<T, 103>, g, b, sm, s, m, st, fp, bp, tm, q_in, kind, lts, fin, keep_delu, flags, with_dt);
  else if (sch == 6)
    launch_ks(m, k_tile_stage<T, 6>, g, b, sm, s, m, st, fp, bp, tm, q_in, kind, lts, fin, keep_delu, flags, with_dt);
  else if (sch == 7)
    launch_ks(m, k_tile_stage<T, 7>, g, b, sm, s, m, st, fp, bp, tm, q_in, kind, lts, fin, keep_delu, flags, with_dt);
  else if (sch == 8)
    launch_ks(m, k_tile_stage<T, 8>, g, b, sm, s, m, st, fp, bp, tm, q_in, kind, lts, fin, keep_delu, flags, with_dt);
  else
    launch_ks(m, k_tile_stage<T, 3>, g, b, sm, s, m, st, fp, bp, tm, q_in, kind, lts, fin, keep_delu, flags, with_dt);
}

int launch_tile_stage(cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp, const BcParams &bp,
                      const TileMesh &tm, const double4 *q_in, int kind, int lts, int fuse_final, int keep_delu,
                      int flags, int with_dt) {
  if (fp.precision == 1)
    launch_tile_t<float>(s, m, st, fp, bp, tm, q_in, kind, lts, fuse_final, keep_delu, flags, with_dt);
  else
    launch_tile_t<double>(s, m, st, fp, bp, tm, q_in, kind, lts, fuse_final, keep_delu, flags, with_dt);
  return 1;
}

template <typename T, bool PRE, int NTHR>
int tile_tma_prepare_t() {
  const int n = static_cast<int>(TileTmaLayout<T, PRE>::bytes);
  const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
  return cudaFuncSetAttribute(k_tile_tma<T, 3, PRE, NTHR>, a, n) == cudaSuccess &&
         cudaFuncSetAttribute(k_tile_tma<T, 103, PRE, NTHR>, a, n) == cudaSuccess &&
         cudaFuncSetAttribute(k_tile_tma<T, 6, PRE, NTHR>, a, n) == cudaSuccess &&
         cudaFuncSetAttribute(k_tile_tma<T, 7, PRE, NTHR>, a, n) == cudaSuccess &&
         cudaFuncSetAttribute(k_tile_tma<T, 8, PRE, NTHR>, a, n) == cudaSuccess;
}

int tile_tma_prepare() {
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
  if (TileTmaLayout<double, true>::bytes > (unsigned)optin) return 0;
  const int ok = tile_tma_prepare_t<double, true, kTileThreadsWide>() &&
                 tile_tma_prepare_t<float, true, kTileThreadsWide>() &&
                 tile_tma_prepare_t<double, true, kTileX * kTileY>() &&
                 tile_tma_prepare_t<float, true, kTileX * kTileY>() &&
                 tile_tma_prepare_t<double, false, kTileX * kTileY>() &&
                 tile_tma_prepare_t<float, false, kTileX * kTileY>();
  cudaGetLastError();
  return ok;
}

void tile_tma_boxes(int q[3], int gw[3], int gs[3]) {
  q[0] = 4;
  q[1] = kTileQW;
  q[2] = kTileQH;
  gw[0] = kTmaRecD;
  gw[1] = kTmaGW;
  gw[2] = kTmaGH;
  gs[0] = kTmaRecD;
  gs[1] = kTmaSW;
  gs[2] = kTmaSH;
}

template <typename T, bool PRE, int NTHR>
void launch_tile_tma_t(cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp, const BcParams &bp,
                       const TileMesh &tm, const TileMaps &maps, const double4 *q_in, int kind, int lts, int fin,
                       int keep_delu, int flags, int with_dt) {
  const unsigned g = static_cast<unsigned>(tm.tiles_i) * static_cast<unsigned>(tm.tiles_j);
  const size_t sm = TileTmaLayout<T, PRE>::bytes;
  const int sch = face_scheme(fp);
  int ahead = 0;
  if (tm.prefetch_ahead) {
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tile_tma<T, 3, PRE, NTHR>, NTHR, sm) == cudaSuccess)
      ahead = sms * per_sm;
    cudaGetLastError();
  }
  if (sch == 103)
    launch_ks(m, k_tile_tma<T, 103, PRE, NTHR>, g, NTHR, sm, s, m, st, fp, bp, tm, maps, q_in, kind, lts, fin,
              keep_delu, flags, with_dt, ahead);
  else if (sch == 6)
    launch_ks(m, k_tile_tma<T, 6, PRE, NTHR>, g, NTHR, sm, s, m, st, fp, bp, tm, maps, q_in, kind, lts, fin, keep_delu,
              flags, with_dt, ahead);
  else if (sch == 7)
    launch_ks(m, k_tile_tma<T, 7, PRE, NTHR>, g, NTHR, sm, s, m, st, fp, bp, tm, maps, q_in, kind, lts, fin, keep_delu,
              flags, with_dt, ahead);
  else if (sch == 8)
    launch_ks(m, k_tile_tma<T, 8, PRE, NTHR>, g, NTHR, sm, s, m, st, fp, bp, tm, maps, q_in, kind, lts, fin, keep_delu,
              flags, with_dt, ahead);
  else
    launch_ks(m, k_tile_tma<T, 3, PRE, NTHR>, g, NTHR, sm, s, m, st, fp, bp, tm, maps, q_in, kind, lts, fin, keep_delu,
              flags, with_dt, ahead);
}

template <typename T>
void launch_tile_tma_v(cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp, const BcParams &bp,
                       const TileMesh &tm, const TileMaps &maps, const double4 *q_in, int kind, int lts, int fin,
                       int keep_delu, int flags, int with_dt, int variant) {
  if (variant == 1)
    launch_tile_tma_t<T, false, kTileX * kTileY>(s, m, st, fp, bp, tm, maps, q_in, kind, lts, fin, keep_delu, flags,
                                                 with_dt);
  else if (variant == 2)
    launch_tile_tma_t<T, true, kTileThreadsWide>(s, m, st, fp, bp, tm, maps, q_in, kind, lts, fin, keep_delu, flags,
                                                 with_dt);
  else
    launch_tile_tma_t<T, true, kTileX * kTileY>(s, m, st, fp, bp, tm, maps, q_in, kind, lts, fin, keep_delu, flags,
                                                with_dt);
}

int launch_tile_tma(cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp, const BcParams &bp,
                    const TileMesh &tm, const TileMaps &maps, const double4 *q_in, int kind, int lts, int fuse_final,
                    int keep_delu, int flags, int with_dt, int variant) {
  if (fp.precision == 1)
    launch_tile_tma_v<float>(s, m, st, fp, bp, tm, maps, q_in, kind, lts, fuse_final, keep_delu, flags, with_dt,
                             variant);
  else
    launch_tile_tma_v<double>(s, m, st, fp, bp, tm, maps, q_in, kind, lts, fuse_final, keep_delu, flags, with_dt,
                              variant);
  return 1;
}

size_t patch_smem_bytes(const DevMesh &m) {
  return sizeof(double) * (12 * (size_t)m.patch_rows + 16 * (size_t)kPatchCells);
}

int patch_prepare(const DevMesh &m) {
  const size_t bytes = patch_smem_bytes(m);
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return 0;
  if (bytes + 4096 > (size_t)optin) return 0;
  const int n = static_cast<int>(bytes);
  if (cudaFuncSetAttribute(k_patch_stage<103>, cudaFuncAttributeMaxDynamicSharedMemorySize, n) != cudaSuccess ||
      cudaFuncSetAttribute(k_patch_stage<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, n) != cudaSuccess ||
      cudaFuncSetAttribute(k_patch_stage<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, n) != cudaSuccess ||
      cudaFuncSetAttribute(k_patch_stage<7>, cudaFuncAttributeMaxDynamicSharedMemorySize, n) != cudaSuccess ||
      cudaFuncSetAttribute(k_patch_stage<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, n) != cudaSuccess)
    return 0;
  return 1;
}

int launch_patch_stage(cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp, const BcParams &bp,
                       int kind, int lts, int fuse_final, int keep_delu, int flags, const double *prim_in) {
  const size_t sm = patch_smem_bytes(m);
  const int g = m.npatch;
  if (face_scheme(fp) == 103)
    launch_ks(m, k_patch_stage<103>, g, kPatchCells, sm, s, m, st, fp, bp, kind, lts, fuse_final, keep_delu, flags,
              prim_in);
  else if (fp.dissipation == 6)
    launch_ks(m, k_patch_stage<6>, g, kPatchCells, sm, s, m, st, fp, bp, kind, lts, fuse_final, keep_delu, flags,
              prim_in);
  else if (fp.dissipation == 7)
    launch_ks(m, k_patch_stage<7>, g, kPatchCells, sm, s, m, st, fp, bp, kind, lts, fuse_final, keep_delu, flags,
              prim_in);
  else if (fp.dissipation == 8)
    launch_ks(m, k_patch_stage<8>, g, kPatchCells, sm, s, m, st, fp, bp, kind, lts, fuse_final, keep_delu, flags,
              prim_in);
  else
    launch_ks(m, k_patch_stage<3>, g, kPatchCells, sm, s, m, st, fp, bp, kind, lts, fuse_final, keep_delu, flags,
              prim_in);
  return 1;
}

int launch_error(cudaStream_t s, const DevMesh &m, DevState &st) {
  k_error<<<nblk(m.NP, kBlock), kBlock, 0, s>>>(m, st);
  return 1;
}

int launch_eval_limiter(cudaStream_t s, int limiter, const double *a, const double *b, int n, double *out) {
  if (n <= 0) return 0;
  k_eval_limiter<<<nblk(n, kBlock), kBlock, 0, s>>>(limiter, a, b, n, out);
  return 1;
}

int launch_eval_face_flux(cudaStream_t s, int scheme, int precision, const double *UL, const double *UR,
                          const double *nrm, const double *len, int n, double *F) {
  if (n <= 0) return 0;
  if (precision == 1) k_eval_face_flux<float><<<nblk(n, kBlock), kBlock, 0, s>>>(scheme, UL, UR, nrm, len, n, F);
  else k_eval_face_flux<double><<<nblk(n, kBlock), kBlock, 0, s>>>(scheme, UL, UR, nrm, len, n, F);
  return 1;
}

int launch_update(cudaStream_t s, const DevMesh &m, DevState &st, int from_S) {
  k_update<<<nblk(m.NP, kBlock), kBlock, 0, s>>>(m, st, from_S);
  return 1;
}

int launch_gradient(cudaStream_t s, const DevMesh &m, DevState &st, int var, double *grad) {
  k_gradient<<<nblk(m.NP, kBlock), kBlock, 0, s>>>(m, st, var, grad);
  return 1;
}

template <typename T, int DISS>
void persistent_kernel_ptr(void (**k)(DevMesh, DevState, FluxParams, BcParams, int, int, int, int, int, int, int,
                                      unsigned int),
                           int minb) {
  if (minb == 0) minb = std::is_same<T, float>::value ? 8 : 6;  // the faster budget of each form on B200
  *k = minb == 8 ? k_persistent_stage<T, DISS, 8>
                  : minb == 6 ? k_persistent_stage<T, DISS, 6> : k_persistent_stage<T, DISS, 4>;
}

// Largest co-resident grid of the persistent stage kernel on this device (0: not available).
int persistent_grid(const FluxParams &fp) {
  void (*k)(DevMesh, DevState, FluxParams, BcParams, int, int, int, int, int, int, int, unsigned int) = nullptr;
  const bool f32 = fp.precision == 1;
  switch (face_scheme(fp)) {
    case 103: f32 ? persistent_kernel_ptr<float, 103>(&k, fp.persist_minb) : persistent_kernel_ptr<double, 103>(&k, fp.persist_minb); break;
    case 6: f32 ? persistent_kernel_ptr<float, 6>(&k, fp.persist_minb) : persistent_kernel_ptr<double, 6>(&k, fp.persist_minb); break;
    case 7: f32 ? persistent_kernel_ptr<float, 7>(&k, fp.persist_minb) : persistent_kernel_ptr<double, 7>(&k, fp.persist_minb); break;
    case 8: f32 ? persistent_kernel_ptr<float, 8>(&k, fp.persist_minb) : persistent_kernel_ptr<double, 8>(&k, fp.persist_minb); break;
    default: f32 ? persistent_kernel_ptr<float, 3>(&k, fp.persist_minb) : persistent_kernel_ptr<double, 3>(&k, fp.persist_minb); break;
  }
  int dev = 0, sms = 0, per_sm = 0, coop = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kPersistBlock, 0) != cudaSuccess) return 0;
  return sms * per_sm;
}

int launch_persistent_stage(cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp,
                            const BcParams &bp, int kind, int lts, int fuse_final, int keep_delu, int flags,
                            int with_dt, int with_bc, int grid, unsigned int test_arrivals) {
  void (*k)(DevMesh, DevState, FluxParams, BcParams, int, int, int, int, int, int, int, unsigned int) = nullptr;
  const bool f32 = fp.precision == 1;
  switch (face_scheme(fp)) {
    case 103: f32 ? persistent_kernel_ptr<float, 103>(&k, fp.persist_minb) : persistent_kernel_ptr<double, 103>(&k, fp.persist_minb); break;
    case 6: f32 ? persistent_kernel_ptr<float, 6>(&k, fp.persist_minb) : persistent_kernel_ptr<double, 6>(&k, fp.persist_minb); break;
    case 7: f32 ? persistent_kernel_ptr<float, 7>(&k, fp.persist_minb) : persistent_kernel_ptr<double, 7>(&k, fp.persist_minb); break;
    case 8: f32 ? persistent_kernel_ptr<float, 8>(&k, fp.persist_minb) : persistent_kernel_ptr<double, 8>(&k, fp.persist_minb); break;
    default: f32 ? persistent_kernel_ptr<float, 3>(&k, fp.persist_minb) : persistent_kernel_ptr<double, 3>(&k, fp.persist_minb); break;
  }
  DevMesh mm = m;
  DevState ss = st;
  FluxParams ff = fp;
  BcParams bb = bp;
  void *args[] = {&mm, &ss, &ff, &bb, &kind, &lts, &fuse_final, &keep_delu, &flags, &with_dt, &with_bc, &test_arrivals};
  cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(k), dim3(grid), dim3(kPersistBlock), args, 0, s);
  return 1;
}

int launch_muscl_gradients(cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp, int with_dt,
                           const BcParams *bc) {
  const int g = m.rblk ? m.n_rblk : nblk(m.NT, kBlock);
  if (m.rblk && g == 0) return 0;
  const BcParams bp = bc ? *bc : BcParams{};
  const int with_bc = bc ? 1 : 0;
  if (with_dt) launch_k(m, k_muscl_gradients<true>, g, kBlock, s, m, st, fp, bp, with_bc);
  else launch_k(m, k_muscl_gradients<false>, g, kBlock, s, m, st, fp, bp, with_bc);
  return 1;
}

int launch_amr_indicator(cudaStream_t s, const DevMesh &m, DevState &st, double *ind) {
  k_amr_indicator<<<nblk(m.NP, kBlock), kBlock, 0, s>>>(m, st, ind);
  return 1;
}

int launch_import_aos(cudaStream_t s, const double *aos, const int *perm, int NP, int NT, double *U) {
  k_import_aos<<<nblk(NT, kBlock), kBlock, 0, s>>>(aos, perm, NP, NT, U);
  return 1;
}

int launch_export_aos(cudaStream_t s, const double *U, const int *perm, int NP, int NT, int ld, double *aos) {
  k_export_aos<<<nblk(NT, kBlock), kBlock, 0, s>>>(U, perm, NP, NT, ld, aos);
  return 1;
}

int launch_amr_tags(cudaStream_t s, const double *ind, const int *ref, int NP, double threshold, double max_fraction,
                    void *scratch, uint8_t *tags) {
  // scratch: two SelectState + 256 histogram counters
  SelectState *sel = reinterpret_cast<SelectState *>(scratch);
  SelectState *sel_ref = sel + 1;
  unsigned int *hist = reinterpret_cast<unsigned int *>(sel + 2);
  const bool top = max_fraction > 0.0 && max_fraction < 1.0;
  int n = 0;
  if (top) {
    long long nRefine = static_cast<long long>(max_fraction * NP);
    if (nRefine < 1) nRefine = 1;
    SelectState init[2] = {{0ull, 0ull, nRefine, 0}, {0ull, 0ull, 0, 0}};
    cudaMemcpyAsync(sel, init, sizeof(init), cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(hist, 0, 256 * sizeof(unsigned int), s);
    const int g = nblk(NP, kBlock) < 1184 ? nblk(NP, kBlock) : 1184;
    for (int shift = 56; shift >= 0; shift -= 8) {
      k_amr_hist<<<g, kBlock, 0, s>>>(ind, ref, NP, sel, shift, 0, 0ull, hist);
      k_amr_pick<<<1, 32, 0, s>>>(sel, shift, 0, hist);
      n += 2;
    }
    // Among the cells whose key equals the cut value, the `remaining` lowest reference ids.
    // The key to match is read on the device inside k_amr_hist via sel_ref->... so copy it.
    SelectState host_sel;
    cudaMemcpyAsync(&host_sel, sel, sizeof(host_sel), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    SelectState init_ref = {0ull, 0xffffffff00000000ull, host_sel.remaining, 0};
    cudaMemcpyAsync(sel_ref, &init_ref, sizeof(init_ref), cudaMemcpyHostToDevice, s);
    for (int shift = 24; shift >= 0; shift -= 8) {
      k_amr_hist<<<g, kBlock, 0, s>>>(ind, ref, NP, sel_ref, shift, 1, host_sel.prefix, hist);
      k_amr_pick<<<1, 32, 0, s>>>(sel_ref, shift, 1, hist);
      n += 2;
    }
  }
  k_amr_tag<<<nblk(NP, kBlock), kBlock, 0, s>>>(ind, ref, NP, threshold, top ? 1 : 0, sel, sel_ref, tags);
  return n + 1;
}

int launch_set_ctl(cudaStream_t s, DevState &st, int idx, double v) {
  k_set_ctl<<<1, 1, 0, s>>>(st.ctl, idx, v);
  return 1;
}

}  // namespace cfdb
