// Host runtime of the C ABI (include/cfd_b200.h): mesh API, device upload / reorder layer,
// stage sequencing, CUDA-graph replay of whole pseudo-steps, downloads.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/cfd_b200.h"
#include "kernels.cuh"
#include "mesh.hpp"
#include "physics.cuh"

namespace cfdb {
std::string config_from_json(const std::string &text, cfd_config *cfg);
void set_last_error(const std::string &msg);
}

using namespace cfdb;

namespace {
thread_local std::string g_err;  // last error message of the calling thread
}  // namespace

void cfdb::set_last_error(const std::string &msg) { g_err = msg; }

namespace {

cfd_status fail(cfd_status s, const std::string &msg) {
  g_err = msg;
  return s;
}

// Tiled tensor map of a 3-D array of doubles (d0 contiguous doubles per element, then d1, then
// d2; rows packed) with box extents box[3], zeros for out-of-range elements.  The encoder is the
// driver's cuTensorMapEncodeTiled, fetched through the runtime (no link to the driver library).
// False when the driver does not offer it or refuses the map.
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn lookup_encode_tiled() {
  void *f = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !f) {
    cudaGetLastError();
    return nullptr;
  }
  return reinterpret_cast<EncodeTiledFn>(f);
}
bool encode_tensor_3d(CUtensorMap *map, const void *base, int d0, int d1, int d2, const int box[3]) {
  static const EncodeTiledFn fn = lookup_encode_tiled();  // looked up once (thread-safe initialisation)
  if (!fn) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)d0, (cuuint64_t)d1, (cuuint64_t)d2};
  const cuuint64_t strides[2] = {(cuuint64_t)d0 * 8, (cuuint64_t)d0 * 8 * d1};
  const cuuint32_t bx[3] = {(cuuint32_t)box[0], (cuuint32_t)box[1], (cuuint32_t)box[2]};
  const cuuint32_t es[3] = {1, 1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void *>(base), dims, strides, bx, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

#define CUDA_TRY(expr)                                                                              \
  do {                                                                                              \
    cudaError_t _e = (expr);                                                                        \
    if (_e != cudaSuccess) return fail(CFD_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)

std::vector<int> rcm_from_arrays(int NP, const int *nf, const int *nbr) {
  std::vector<int> deg(NP, 0);
  for (int c = 0; c < NP; c++)
    for (int f = 0; f < nf[c]; f++)
      if (nbr[4 * c + f] >= 0 && nbr[4 * c + f] < NP) deg[c]++;
  std::vector<int> by_deg(NP);
  for (int i = 0; i < NP; i++) by_deg[i] = i;
  std::stable_sort(by_deg.begin(), by_deg.end(), [&](int a, int b) { return deg[a] < deg[b]; });
  std::vector<int> order;
  order.reserve(NP);
  std::vector<char> seen(NP, 0);
  std::vector<int> q, nb;
  q.reserve(NP);
  for (int start : by_deg) {
    if (seen[start]) continue;
    size_t head = q.size();
    q.push_back(start);
    seen[start] = 1;
    while (head < q.size()) {
      int c = q[head++];
      order.push_back(c);
      nb.clear();
      for (int f = 0; f < nf[c]; f++) {
        int n = nbr[4 * c + f];
        if (n >= 0 && n < NP && !seen[n]) nb.push_back(n);
      }
      std::stable_sort(nb.begin(), nb.end(), [&](int a, int b) { return deg[a] < deg[b]; });
      for (int n : nb) {
        seen[n] = 1;
        q.push_back(n);
      }
    }
  }
  std::reverse(order.begin(), order.end());
  return order;
}

// Patch ordering: cells grouped into patches of `patch` cells grown breadth-first from seeds
// taken in RCM order, so a thread block of `patch` cells covers a compact piece of the mesh and
// most of its neighbours lie inside the same block (cache reuse for the gather kernels).
std::vector<int> patch_from_arrays(int NP, const int *nf, const int *nbr, int patch) {
  const std::vector<int> rcm = rcm_from_arrays(NP, nf, nbr);
  std::vector<char> used(NP, 0);
  std::vector<int> order, q;
  order.reserve(NP);
  q.reserve(patch);
  for (int seed : rcm) {
    if (used[seed]) continue;
    q.clear();
    q.push_back(seed);
    used[seed] = 1;
    for (size_t head = 0; head < q.size(); head++) {
      const int c = q[head];
      order.push_back(c);
      for (int f = 0; f < nf[c]; f++) {
        const int n = nbr[4 * c + f];
        if (n >= 0 && n < NP && !used[n] && (int)q.size() < patch) {
          used[n] = 1;
          q.push_back(n);
        }
      }
    }
  }
  return order;
}

// Patch ordering by recursive coordinate bisection, for the one-block-per-patch stage kernel.
// Cell centres are recovered (up to a shift per connected piece of the mesh) by walking the face
// graph with the centre-to-centre vectors; each piece is then cut at the median of its longer
// extent until every part has at most `patch` cells, the cuts chosen so that all parts of a piece
// but the last hold exactly `patch` cells.  Parts are numbered depth-first (neighbouring parts get
// nearby numbers); the cells of a part keep their given order.  starts[b] = first cell of part b.
void rcb_patches(int NP, const int *nf, const int *nbr, const double *cvec, int patch, std::vector<int> &order,
                 std::vector<int> &starts) {
  std::vector<double> x(NP, 0.0), y(NP, 0.0);
  std::vector<char> seen(NP, 0);
  std::vector<int> comp, q;
  order.clear();
  starts.clear();
  order.reserve(NP);
  q.reserve(NP);
  auto split = [&](auto &&self, int lo, int hi) -> void {
    const int n = hi - lo;
    if (n <= patch) {
      std::sort(comp.begin() + lo, comp.begin() + hi);
      starts.push_back(static_cast<int>(order.size()));
      order.insert(order.end(), comp.begin() + lo, comp.begin() + hi);
      return;
    }
    double xmin = 1e300, xmax = -1e300, ymin = 1e300, ymax = -1e300;
    for (int i = lo; i < hi; i++) {
      const int c = comp[i];
      xmin = std::min(xmin, x[c]);
      xmax = std::max(xmax, x[c]);
      ymin = std::min(ymin, y[c]);
      ymax = std::max(ymax, y[c]);
    }
    const std::vector<double> &a = (xmax - xmin >= ymax - ymin) ? x : y;
    const int k = (n + patch - 1) / patch;
    const int left = (k / 2) * patch;
    std::nth_element(comp.begin() + lo, comp.begin() + lo + left, comp.begin() + hi,
                     [&](int u, int v) { return a[u] < a[v] || (a[u] == a[v] && u < v); });
    self(self, lo, lo + left);
    self(self, lo + left, hi);
  };
  for (int s0 = 0; s0 < NP; s0++) {
    if (seen[s0]) continue;
    q.clear();
    q.push_back(s0);
    seen[s0] = 1;
    for (size_t h = 0; h < q.size(); h++) {
      const int c = q[h];
      for (int f = 0; f < nf[c]; f++) {
        const int n = nbr[4 * c + f];
        if (n < 0 || n >= NP || seen[n]) continue;
        seen[n] = 1;
        x[n] = x[c] + cvec[8 * c + 2 * f];
        y[n] = y[c] + cvec[8 * c + 2 * f + 1];
        q.push_back(n);
      }
    }
    comp = q;
    split(split, 0, static_cast<int>(comp.size()));
  }
}

// Structured-block numbering (reorder 4): recognises a mesh that is one block of ni x nj quads
// (every cell a quad, one corner cell with ghosts on two adjacent faces, straight lines of faces
// from it) and numbers its cells c = j * ni + i.  Walking from a cell c through face slot s to its
// neighbour n continues straight through the slot opposite the one of n that faces c (slot + 2:
// the four faces of a quad are stored in order around it).  The i direction is the one whose
// length is a multiple of the tile width if only one is, else the longer one.  Per cell the slot
// of +i (E) and +j (N); lh = 1 when the slot after E is S (clockwise slot order in (i, j)).
struct BlockOrder {
  int ni = 0, nj = 0, lh = 0;
  std::vector<int> cell;     // [nj * ni] reference cell of (i, j)
  std::vector<int> sE, sN;   // per reference cell: slot of its +i and +j faces
};

bool structured_block(int NP, const int *nf, const int *nbr, BlockOrder &b, std::string &why) {
  auto phys = [&](int n) { return n >= 0 && n < NP; };
  auto back = [&](int n, int c) {
    for (int k = 0; k < 4; k++)
      if (nbr[4 * n + k] == c) return k;
    return -1;
  };
  for (int c = 0; c < NP; c++)
    if (nf[c] != 4) {
      why = "cell " + std::to_string(c) + " is not a quad";
      return false;
    }
  int c0 = -1, fa = -1, fb = -1;
  for (int c = 0; c < NP && c0 < 0; c++)
    for (int f = 0; f < 4; f++)
      if (!phys(nbr[4 * c + f]) && !phys(nbr[4 * c + ((f + 1) & 3)]) && phys(nbr[4 * c + ((f + 2) & 3)]) &&
          phys(nbr[4 * c + ((f + 3) & 3)])) {
        c0 = c;
        fa = (f + 2) & 3;
        fb = (f + 3) & 3;
        break;
      }
  if (c0 < 0) {
    why = "no corner cell (a cell with ghosts on two adjacent faces)";
    return false;
  }
  auto walk = [&](int c, int s) {
    int len = 1;
    while (len <= NP) {
      const int n = nbr[4 * c + s];
      if (!phys(n)) return len;
      const int g = back(n, c);
      if (g < 0) return -1;
      s = (g + 2) & 3;
      c = n;
      len++;
    }
    return -1;
  };
  const int la = walk(c0, fa), lb = walk(c0, fb);
  if (la < 2 || lb < 2) {
    why = "the block is thinner than two cells";
    return false;
  }
  const bool a32 = la % 32 == 0, b32 = lb % 32 == 0;
  const bool a_is_i = (a32 != b32) ? a32 : la >= lb;
  b.ni = a_is_i ? la : lb;
  b.nj = a_is_i ? lb : la;
  const int si = a_is_i ? fa : fb, sj = a_is_i ? fb : fa;
  if ((long long)b.ni * b.nj != NP) {
    why = "the lines from the corner cell span " + std::to_string(b.ni) + " x " + std::to_string(b.nj) + " cells, not " +
          std::to_string(NP);
    return false;
  }
  const int h = (si - sj) & 3;  // slot(E) - slot(N)
  b.lh = h == 1;
  b.cell.assign((size_t)NP, -1);
  b.sE.assign(NP, -1);
  b.sN.assign(NP, -1);
  int rowc = c0, rows = sj;
  for (int j = 0; j < b.nj; j++) {
    if (j > 0) {
      const int n = nbr[4 * rowc + rows];
      const int g = phys(n) ? back(n, rowc) : -1;
      if (g < 0) {
        why = "column walk leaves the block at row " + std::to_string(j);
        return false;
      }
      rows = (g + 2) & 3;
      rowc = n;
    }
    int c = rowc, se = (rows + h) & 3;
    for (int i = 0; i < b.ni; i++) {
      if (i > 0) {
        const int n = nbr[4 * c + se];
        const int g = phys(n) ? back(n, c) : -1;
        if (g < 0) {
          why = "row walk leaves the block at (" + std::to_string(i) + ", " + std::to_string(j) + ")";
          return false;
        }
        se = (g + 2) & 3;
        c = n;
      }
      if (b.sE[c] >= 0) {
        why = "cell " + std::to_string(c) + " is reached twice";
        return false;
      }
      b.cell[(size_t)j * b.ni + i] = c;
      b.sE[c] = se;
      b.sN[c] = (se - h) & 3;
    }
  }
  // Every neighbour relation must be the block's: (i +- 1, j), (i, j +- 1), or a ghost on the rim.
  for (int j = 0; j < b.nj; j++)
    for (int i = 0; i < b.ni; i++) {
      const int c = b.cell[(size_t)j * b.ni + i];
      const int want[4] = {i + 1 < b.ni ? b.cell[(size_t)j * b.ni + i + 1] : -1,
                           j + 1 < b.nj ? b.cell[(size_t)(j + 1) * b.ni + i] : -1,
                           i > 0 ? b.cell[(size_t)j * b.ni + i - 1] : -1, j > 0 ? b.cell[(size_t)(j - 1) * b.ni + i] : -1};
      const int slot[4] = {b.sE[c], b.sN[c], (b.sE[c] + 2) & 3, (b.sN[c] + 2) & 3};
      for (int q = 0; q < 4; q++) {
        const int n = nbr[4 * c + slot[q]];
        if (want[q] >= 0 ? n != want[q] : phys(n)) {
          why = "cell (" + std::to_string(i) + ", " + std::to_string(j) + ") does not neighbour the block's cells";
          return false;
        }
      }
    }
  return true;
}

template <typename T>
cfd_status dev_upload(T **dst, const std::vector<T> &v) {
  CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(dst), std::max<size_t>(1, v.size()) * sizeof(T)));
  if (!v.empty()) CUDA_TRY(cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return CFD_OK;
}
}  // namespace

struct cfd_mesh {
  Mesh m;
};

struct cfd_ctx {
  cfd_config cfg{};
  int NP = 0, NG = 0, NT = 0, NB = 0;
  std::vector<int> perm;  // device index -> reference index (physical)
  std::vector<int> inv;   // reference index -> device index (physical)
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  DevMesh dm{};
  DevState ds{};
  FluxParams fp{};
  BcParams bp{};
  std::vector<void *> allocs;
  size_t bytes = 0;
  long long launches = 0;
  bool prim_from_S = false;
  int keep_delu = 1;
  int use_graph = 1;
  int fuse_gather = 1;  // face-based forms with per-cell dt: fused gather + stage update
  int patch_stage = 0;  // ... or, with patch tables (reorder 3), the one-kernel patch stage
  bool ghost_private = false;  // every ghost row has one boundary entry and neighbours only its owner
  size_t l2_window = 0;        // bytes of the face-flux L2 window (option "l2_persist" turns it on/off)
  std::vector<int> patch_starts;  // first device cell of each patch (reorder 3)
  double *pbuf[2] = {nullptr, nullptr};  // stage primitives of the patch form ([5][NT] each)
  cudaGraphExec_t graph = nullptr;
  int graph_launches = 0;
  // Persistent batched form (option "persistent"): one cooperative launch per RK stage, one
  // CUDA graph per stage; persist_grid = co-resident blocks used; persist_test_arrivals = barrier
  // arrivals that never come (option "barrier_timeout_test", a test of the timeout path).
  bool persistent = false;
  int persist_grid = 0;
  int partial_blocks = 0;  // blocks the reduction buffers (st.partial) are sized for
  unsigned int persist_test_arrivals = 0;
  bool stage_graphs_ok = true;
  cudaGraphExec_t stage_graph[4] = {nullptr, nullptr, nullptr, nullptr};
  int stage_graph_launches[4] = {0, 0, 0, 0};
  int n_stage_graphs = 0;
  double *h_ctl = nullptr;  // pinned mirror of the control block
  int *d_perm = nullptr;    // device copy of perm
  int *d_lf_cells = nullptr;       // Lax_Fedrichs: device cells grouped by wavefront level
  std::vector<int> lf_level_start;  // first entry of each level in d_lf_cells, plus the end
  // Tile form (reorder 4 on a structured block, option "tile_stage"): the block tables and the two
  // further (rho, u, v, p) row buffers the stages of a step rotate through (st.q4 -> qbuf[0] ->
  // qbuf[1] -> st.q4).
  TileMesh tm{};
  bool tile_ok = false;
  // 0 off, 1 the tile kernel, 2 its TMA form (stage inputs prefetched), 3 TMA form with 3 blocks
  // per SM, 4 TMA form with 288 threads
  int tile_stage = 0;
  double4 *qbuf[2] = {nullptr, nullptr};
  // TMA form: tensor maps of the three row buffers (st.q4, qbuf[0], qbuf[1]) and of the two
  // face-record tensors; tile_tma_ok when all of them were encoded.
  bool tile_tma_ok = false;
  CUtensorMap tmap_q[3];
  CUtensorMap tmap_gw, tmap_gs;
  // Per-kernel timing (option "profile"): event pairs recorded around each launch on the
  // context's stream, resolved lazily by cfd_kernel_time.
  int profile = 0;
  struct Timed {
    int kind;
    cudaEvent_t a, b;
  };
  std::vector<Timed> timed;
  double kind_ms[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  long long kind_n[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  double *d_stage = nullptr;  // [NT*4] reference-order AoS staging rows
  void *d_amr = nullptr;      // AMR indicator, tags and selection scratch (allocated on first use)
  int2 *d_tables = nullptr;   // work lists of batched solves (cells, faces, entries, records)
};

namespace {

cfd_status ctx_alloc(cfd_ctx *ctx, void **p, size_t bytes) {
  CUDA_TRY(cudaMalloc(p, std::max<size_t>(bytes, 16)));
  ctx->allocs.push_back(*p);
  ctx->bytes += bytes;
  return CFD_OK;
}

template <typename T>
cfd_status ctx_upload(cfd_ctx *ctx, T **dst, const std::vector<T> &v) {
  cfd_status s = ctx_alloc(ctx, reinterpret_cast<void **>(dst), v.size() * sizeof(T));
  if (s != CFD_OK) return s;
  if (!v.empty()) CUDA_TRY(cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return CFD_OK;
}

int dev_of(const cfd_ctx *ctx, int ref) { return ref < ctx->NP ? ctx->inv[ref] : ref; }

enum { TK_FLUX = 0, TK_STAGE = 1, TK_BC = 2, TK_GRAD = 3, TK_FACES = 4, TK_GATHER_STAGE = 5, TK_PATCH = 6, TK_PERSIST = 7,
       TK_TILE = 8, TK_N = 9 };

struct TimedScope {
  cfd_ctx *ctx;
  int kind;
  cudaEvent_t a = nullptr, b = nullptr;
  TimedScope(cfd_ctx *c, int k) : ctx(c), kind(k) {
    if (!ctx->profile) return;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, ctx->stream);
  }
  ~TimedScope() {
    if (!ctx->profile) return;
    cudaEventRecord(b, ctx->stream);
    ctx->timed.push_back({kind, a, b});
  }
};

// Stage sequence of one pseudo-step for the configured integrator.
struct StagePlan {
  int n;        // stages
  int kind0;    // stage kind of stage 0 (kinds kind0 .. kind0 + n - 1; 0 = explicit)
  int src_S;    // the supersonic-exit copy of stages > 0 reads the stage state
  int lts_mode; // 0: per-stage rule of the reference (LTS in stage 1 only), 1: dt frozen per step
};

StagePlan stage_plan(const cfd_config &c, int consistent) {
  if (c.integrator == CFD_INT_REFERENCE && !c.time_accurate) return {1, 0, 0, 0};
  if (c.integrator == CFD_INT_RK4) return {4, 11, 1, 1};
  if (c.integrator == CFD_INT_RK3_GPU_REF) return {3, 21, 1, 1};
  if (c.integrator == CFD_INT_RK4_GPU_REF) return {4, 31, 1, 1};
  if (c.integrator == CFD_INT_SSPRK3) return {3, 1, consistent, 1};
  return {3, 1, consistent, 0};
}

// lts argument of the stage kernels for stage k (see k_stage).
int stage_lts(const StagePlan &p, const cfd_config &c, int k) {
  if (p.kind0 == 0) return 0;
  if (p.lts_mode == 1) return c.local_time_stepping ? 2 : 3;
  return (k == 0 && c.local_time_stepping) ? 1 : 0;
}

void drop_graphs(cfd_ctx *ctx) {
  if (ctx->graph) cudaGraphExecDestroy(ctx->graph);
  ctx->graph = nullptr;
  for (int k = 0; k < 4; k++) {
    if (ctx->stage_graph[k]) cudaGraphExecDestroy(ctx->stage_graph[k]);
    ctx->stage_graph[k] = nullptr;
  }
  ctx->n_stage_graphs = 0;
}

// Launch sequence of stage k of one pseudo-step (loop body of src/Solver.cpp:94-125): the
// boundary conditions, the residual (face-based forms: gradients, face fluxes, gather) and the
// update.  ghosts_written carries "the previous stage's owner threads wrote this stage's ghosts"
// from stage to stage (false before stage 0).
int enqueue_stage(cfd_ctx *ctx, int k, bool fuse_final, bool &ghosts_written) {
  const cfd_config &c = ctx->cfg;
  cudaStream_t s = ctx->stream;
  DevMesh &m = ctx->dm;
  DevState &st = ctx->ds;
  int n = 0;
  const StagePlan p = stage_plan(c, ctx->fp.consistent);
  const bool faces = ctx->dm.NF > 0;
  // Patch form: one kernel per stage.  Stage k reads the primitives of buffer in(k) and writes
  // out(k): in(0) = st.prim, out(k) = pbuf[k % 2] for the other stages and st.prim for the last,
  // in(k + 1) = out(k), so every stage writes a buffer that no block of it reads.
  const bool patch = faces && ctx->patch_stage && m.npatch > 0 && !m.cblk && !m.fblk && fuse_final &&
                     ctx->fp.precision == CFD_PREC_FP64 && !ctx->fp.weno && p.kind0 != 0 && p.lts_mode == 1 &&
                     c.local_time_stepping;
  // Tile form: one kernel per stage on a structured block; the three stages rotate the
  // (rho, u, v, p) rows through st.q4 -> qbuf[0] -> qbuf[1] -> st.q4 (each stage writes a buffer
  // that no block of it reads), and the step's boundary conditions come from launch_bc.
  const bool tile = faces && ctx->tile_ok && ctx->tile_stage && !m.cblk && !m.fblk && fuse_final && !ctx->fp.weno &&
                    p.n == 3 && p.kind0 != 0 && p.lts_mode == 1 && c.local_time_stepping;
  const int kind = p.kind0 == 0 ? 0 : p.kind0 + k;
  const int lts = stage_lts(p, c, k);
  const int fin = (k == p.n - 1) ? fuse_final : 0;
  // Fused face-based stages take the first stage's boundary conditions into the gradient pass
  // (each cell applies its own entries before its gradient) when no ghost is shared.
  const bool fused_faces = faces && ctx->fuse_gather && (lts == 1 || lts == 2);
  const bool bc_in_grad = fused_faces && !patch && !tile && k == 0 && ctx->ghost_private;
  if (!ghosts_written && !bc_in_grad) {
    TimedScope ts(ctx, TK_BC);
    n += launch_bc(s, m, st, ctx->bp, k > 0 && p.src_S, k > 0);
  }
  ghosts_written = false;
  if (tile) {
    TimedScope ts(ctx, TK_TILE);
    const bool bc_next = k < p.n - 1;
    const int flags = (bc_next ? 2 : 0) | (p.src_S ? 4 : 0);
    double4 *bufs[3] = {st.q4, ctx->qbuf[0], ctx->qbuf[1]};
    DevState sk = st;
    sk.q4 = bufs[(k + 1) % 3];
    const bool with_dt = k == 0 || k == p.n - 1;
    if (ctx->tile_stage >= 2 && ctx->tile_tma_ok) {
      TileMaps maps;
      maps.q = ctx->tmap_q[k];
      maps.gw = ctx->tmap_gw;
      maps.gs = ctx->tmap_gs;
      n += launch_tile_tma(s, m, sk, ctx->fp, ctx->bp, ctx->tm, maps, bufs[k], kind, lts, fin, ctx->keep_delu, flags,
                           with_dt ? 1 : 0, ctx->tile_stage - 2);
    } else {
      n += launch_tile_stage(s, m, sk, ctx->fp, ctx->bp, ctx->tm, bufs[k], kind, lts, fin, ctx->keep_delu, flags,
                             with_dt ? 1 : 0);
    }
    ghosts_written = bc_next;
    return n;
  }
  if (patch) {
    TimedScope ts(ctx, TK_PATCH);
    const bool bc_next = k < p.n - 1;
    const int flags = (bc_next ? 2 : 0) | (p.src_S ? 4 : 0);
    DevState sk = st;
    sk.prim = bc_next ? ctx->pbuf[k % 2] : st.prim;
    const double *pin = k == 0 ? st.prim : ctx->pbuf[(k - 1) % 2];
    n += launch_patch_stage(s, m, sk, ctx->fp, ctx->bp, kind, lts, fin, ctx->keep_delu, flags, pin);
    ghosts_written = bc_next;
    return n;
  }
  if (faces) {
    // Fused form (per-cell dt): del_t comes from the gradient pass, the stage kernel writes
    // the next stage's ghost states from the owner cells, and the last stage forms the step's
    // Min_dt from the per-cell dt frozen at the first stage.
    const bool fused = ctx->fuse_gather && (lts == 1 || lts == 2);
    // del_t is formed where a stage uses it (lts 1, or the first stage, which freezes it) and
    // at the last stage, whose value is the Cells[].del_t a download returns.
    const bool with_dt = fused && (lts == 1 || k == 0 || k == p.n - 1);
    if (fused && ctx->persistent && ctx->persist_grid > 0) {
      TimedScope ts(ctx, TK_PERSIST);
      const bool bc_next = k < p.n - 1;
      const int flags = (bc_next ? 2 : 0) | (p.src_S ? 4 : 0);
      n += launch_persistent_stage(s, m, st, ctx->fp, ctx->bp, kind, lts, fin, ctx->keep_delu, flags, with_dt ? 1 : 0,
                                   bc_in_grad ? 1 : 0, ctx->persist_grid, ctx->persist_test_arrivals);
      ghosts_written = bc_next;
      return n;
    }
    {
      TimedScope ts(ctx, TK_GRAD);
      n += launch_muscl_gradients(s, m, st, ctx->fp, with_dt ? 1 : 0, bc_in_grad ? &ctx->bp : nullptr);
    }
    { TimedScope ts(ctx, TK_FACES); n += launch_faces(s, m, st, ctx->fp); }
    if (fused) {
      TimedScope ts(ctx, TK_GATHER_STAGE);
      const bool bc_next = k < p.n - 1;
      const int flags = (bc_next ? 2 : 0) | (p.src_S ? 4 : 0);
      n += launch_gather_stage(s, m, st, ctx->fp, ctx->bp, kind, lts, fin, ctx->keep_delu, flags);
      ghosts_written = bc_next;
    } else {
      { TimedScope ts(ctx, TK_FLUX); n += launch_gather(s, m, st, ctx->fp); }
      { TimedScope ts(ctx, TK_STAGE); n += launch_stage(s, m, st, kind, lts, fin, ctx->keep_delu); }
    }
    return n;
  }
  { TimedScope ts(ctx, TK_FLUX); n += launch_flux(s, m, st, ctx->fp, k > 0); }
  { TimedScope ts(ctx, TK_STAGE); n += launch_stage(s, m, st, kind, lts, fin, ctx->keep_delu); }
  return n;
}

// Launch sequence of one pseudo-step: its stages in order.
int enqueue_step(cfd_ctx *ctx, bool fuse_final) {
  const StagePlan p = stage_plan(ctx->cfg, ctx->fp.consistent);
  bool ghosts_written = false;
  int n = 0;
  for (int k = 0; k < p.n; k++) n += enqueue_stage(ctx, k, fuse_final, ghosts_written);
  return n;
}

cfd_status sync_status(cfd_ctx *ctx, cfd_step_info *info) {
  CUDA_TRY(cudaMemcpyAsync(ctx->h_ctl, ctx->ds.ctl, sizeof(double) * CTL_SIZE, cudaMemcpyDeviceToHost, ctx->stream));
  int h_status[2];
  CUDA_TRY(cudaMemcpyAsync(h_status, ctx->ds.status, sizeof(h_status), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  CUDA_TRY(cudaGetLastError());
  cfd_status st = static_cast<cfd_status>(h_status[0]);
  int bad = -1;
  if (st == CFD_ERR_NONPHYSICAL && h_status[1] != INT_MAX) {
    bad = h_status[1] < ctx->NP ? ctx->perm[h_status[1]] : h_status[1];
  }
  if (info) {
    info->iterations = static_cast<int>(ctx->h_ctl[CTL_ITER]);
    info->min_dt = ctx->h_ctl[CTL_DTMIN];
    info->total_time = ctx->h_ctl[CTL_TOTAL_TIME];
    for (int k = 0; k < 4; k++) {
      info->error[k] = ctx->h_ctl[CTL_ERR + k];
      info->res_l2[k] = ctx->h_ctl[CTL_RES + k];
    }
    info->bad_cell = bad;
    info->status = st;
  }
  if (st == CFD_ERR_NONPHYSICAL) return fail(st, "non-physical state (NaN sound speed) at cell " + std::to_string(bad));
  if (st != CFD_OK) return fail(st, "device status " + std::to_string(st));
  return CFD_OK;
}

}  // namespace

// ---------------------------------------------------------------------------------------------
extern "C" {

const char *cfd_last_error(void) { return g_err.c_str(); }
const char *cfd_version(void) { return "cfd-b200 0.1 (sm_100a, fp64 exact)"; }

// ----------------------------------------- mesh -------------------------------------------
static cfd_status finish_mesh(cfd_mesh *h, const std::string &gen_err, cfd_mesh **out) {
  if (!gen_err.empty()) {
    delete h;
    return fail(CFD_ERR_MESH, gen_err);
  }
  std::string e = h->m.build();
  if (!e.empty()) {
    delete h;
    return fail(CFD_ERR_MESH, e);
  }
  *out = h;
  return CFD_OK;
}

cfd_status cfd_mesh_block_order(const cfd_mesh_desc *d, int *ni, int *nj, int *lh, int *cells) {
  if (!d || !ni || !nj || !lh || !d->n_faces || !d->neighbours || d->n_physical <= 0)
    return fail(CFD_ERR_BAD_ARG, "bad argument");
  BlockOrder b;
  std::string why;
  if (!structured_block(d->n_physical, d->n_faces, d->neighbours, b, why))
    return fail(CFD_ERR_MESH, "not a single structured block of quads: " + why);
  *ni = b.ni;
  *nj = b.nj;
  *lh = b.lh;
  if (cells) std::copy(b.cell.begin(), b.cell.end(), cells);
  return CFD_OK;
}

cfd_status cfd_mesh_box(int nx, int ny, double x0, double x1, double y0, double y1, cfd_mesh **out) {
  if (!out) return fail(CFD_ERR_BAD_ARG, "null out");
  cfd_mesh *h = new cfd_mesh;
  return finish_mesh(h, generate_box(h->m, nx, ny, x0, x1, y0, y1), out);
}
cfd_status cfd_mesh_half_cylinder(int ntheta, int nr, double r_body, double r_outer, double ratio, cfd_mesh **out) {
  if (!out) return fail(CFD_ERR_BAD_ARG, "null out");
  cfd_mesh *h = new cfd_mesh;
  return finish_mesh(h, generate_half_cylinder(h->m, ntheta, nr, r_body, r_outer, ratio), out);
}
cfd_status cfd_mesh_ramp(int nx, int ny, double length, double height, double x_corner, double angle_deg,
                         int open_top, cfd_mesh **out) {
  if (!out) return fail(CFD_ERR_BAD_ARG, "null out");
  cfd_mesh *h = new cfd_mesh;
  return finish_mesh(h, generate_ramp(h->m, nx, ny, length, height, x_corner, angle_deg, open_top), out);
}
cfd_status cfd_mesh_bump(int nx, int ny, double length, double height, double thickness, int n_quad_layers,
                         double jitter, uint64_t seed, int triangles, cfd_mesh **out) {
  if (!out) return fail(CFD_ERR_BAD_ARG, "null out");
  cfd_mesh *h = new cfd_mesh;
  return finish_mesh(h, generate_bump(h->m, nx, ny, length, height, thickness, n_quad_layers, jitter, seed, triangles),
                     out);
}
cfd_status cfd_mesh_read_vtk(const char *path, cfd_mesh **out) {
  if (!out || !path) return fail(CFD_ERR_BAD_ARG, "null argument");
  cfd_mesh *h = new cfd_mesh;
  std::string e = read_vtk(h->m, path);
  if (!e.empty()) {
    delete h;
    return fail(CFD_ERR_IO, e);
  }
  return finish_mesh(h, "", out);
}
cfd_status cfd_mesh_write_vtk(const cfd_mesh *m, const char *path) {
  if (!m || !path) return fail(CFD_ERR_BAD_ARG, "null argument");
  std::string e = write_vtk(m->m, path);
  return e.empty() ? CFD_OK : fail(CFD_ERR_IO, e);
}
cfd_status cfd_mesh_describe(const cfd_mesh *h, cfd_mesh_desc *d) {
  if (!h || !d) return fail(CFD_ERR_BAD_ARG, "null argument");
  const Mesh &m = h->m;
  d->n_physical = m.n_physical;
  d->n_ghost = m.n_ghost;
  d->n_faces = m.n_faces.data();
  d->neighbours = m.nbr.data();
  d->face_normals = m.normals.data();
  d->face_lengths = m.lengths.data();
  d->center_distances = m.ccd.data();
  d->center_vectors = m.cvec.data();
  d->area = m.area.data();
  d->inv_area = m.inv_area.data();
  d->n_boundary = static_cast<int>(m.boundary.size() / 4);
  d->boundary = m.boundary.data();
  return CFD_OK;
}
cfd_status cfd_mesh_centers(const cfd_mesh *h, double *out) {
  if (!h || !out) return fail(CFD_ERR_BAD_ARG, "null argument");
  std::memcpy(out, h->m.centers.data(), h->m.centers.size() * sizeof(double));
  return CFD_OK;
}
cfd_status cfd_mesh_points(const cfd_mesh *h, int *n_points, const double **points) {
  if (!h || !n_points || !points) return fail(CFD_ERR_BAD_ARG, "null argument");
  *n_points = static_cast<int>(h->m.points.size() / 3);
  *points = h->m.points.data();
  return CFD_OK;
}
void cfd_mesh_destroy(cfd_mesh *m) { delete m; }

// ----------------------------------------- config -----------------------------------------
void cfd_config_default(cfd_config *c) {
  std::memset(c, 0, sizeof(*c));
  c->dissipation_type = CFD_DISS_ROE;
  c->is_second_order = 1;
  c->time_accurate = 0;
  c->local_time_stepping = 0;
  c->integrator = CFD_INT_REFERENCE;
  c->limiter = CFD_LIM_REF_MINMOD;
  c->cfl = 0.1;
  c->limiter_zeta = 0.5;
  c->limiter_zeta1 = 0.5;
  c->inlet_rho = 1.0;
  c->inlet_p = 1.0 / 1.4;
  c->r_gas = 287.0;
  c->reorder = 1;
}

cfd_status cfd_config_read_json(const char *path, cfd_config *cfg) {
  if (!path || !cfg) return fail(CFD_ERR_BAD_ARG, "null argument");
  std::ifstream in(path);
  if (!in) return fail(CFD_ERR_IO, std::string("cannot open ") + path);
  std::stringstream ss;
  ss << in.rdbuf();
  std::string e = config_from_json(ss.str(), cfg);
  return e.empty() ? CFD_OK : fail(CFD_ERR_BAD_ARG, "JSON: " + e);
}

// ----------------------------------------- context ----------------------------------------
void cfd_destroy(cfd_ctx *ctx) {
  if (!ctx) return;
  drop_graphs(ctx);
  for (auto &t : ctx->timed) {
    cudaEventDestroy(t.a);
    cudaEventDestroy(t.b);
  }
  for (void *p : ctx->allocs) cudaFree(p);
  if (ctx->h_ctl) cudaFreeHost(ctx->h_ctl);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

cfd_status cfd_create(const cfd_mesh_desc *d, const cfd_config *cfg, cfd_ctx **out) {
  if (!d || !cfg || !out) return fail(CFD_ERR_BAD_ARG, "null argument");
  *out = nullptr;
  const int NP = d->n_physical, NG = d->n_ghost, NB = d->n_boundary;
  if (NP <= 0 || NG < 0 || NB < 0) return fail(CFD_ERR_BAD_ARG, "bad mesh sizes");
  if (!d->n_faces || !d->neighbours || !d->face_normals || !d->face_lengths || !d->area || !d->inv_area ||
      (NB > 0 && !d->boundary))
    return fail(CFD_ERR_BAD_ARG, "missing mesh arrays");
  if (cfg->is_second_order && !d->center_distances) return fail(CFD_ERR_BAD_ARG, "second order needs centre distances");
  const int NT = NP + NG;
  for (int c = 0; c < NP; c++) {
    int nf = d->n_faces[c];
    if (nf != 3 && nf != 4) return fail(CFD_ERR_MESH, "cell " + std::to_string(c) + " must have 3 or 4 faces");
    for (int f = 0; f < nf; f++) {
      int n = d->neighbours[4 * c + f];
      if (n < 0 || n >= NT) return fail(CFD_ERR_MESH, "cell " + std::to_string(c) + " has an invalid neighbour");
    }
  }
  for (int e = 0; e < NB; e++) {
    const int *b = d->boundary + 4 * e;
    if (b[0] < 0 || b[0] > 3 || b[1] < 0 || b[1] >= NP || b[2] < 0 || b[2] >= d->n_faces[b[1]] || b[3] < NP || b[3] >= NT)
      return fail(CFD_ERR_MESH, "invalid boundary entry " + std::to_string(e));
  }
  const int diss = cfg->dissipation_type;
  if (diss < CFD_DISS_LLF || diss > CFD_DISS_AUSM_GPU)
    return fail(CFD_ERR_BAD_ARG, "dissipation type " + std::to_string(diss) + " is not available in this build");
  const bool movers_family = diss == CFD_DISS_MOVERS || diss == CFD_DISS_RICCA || diss == CFD_DISS_MOVERS_NWSC;
  if (movers_family && cfg->is_second_order && cfg->muscl)
    return fail(CFD_ERR_BAD_ARG, "MOVERS, RICCA and MOVERS_NWSC are available in the reference's per-cell form "
                                 "only (muscl = 0)");
  if (movers_family && cfg->is_second_order && cfg->reconstruct_primitive)
    return fail(CFD_ERR_BAD_ARG, "RICCA_2O and MOVERS_NWSC_2O limit the conserved variables (reconstruct_primitive = 0)");
  if (diss == CFD_DISS_AUSM_GPU && !(cfg->is_second_order && cfg->muscl))
    return fail(CFD_ERR_BAD_ARG, "the reference GPU AUSM face flux is available in the gradient-MUSCL form only");
  if (cfg->integrator < CFD_INT_REFERENCE || cfg->integrator > CFD_INT_RK4_GPU_REF)
    return fail(CFD_ERR_BAD_ARG, "bad integrator");
  if (cfg->weno && cfg->muscl && cfg->is_second_order)
    return fail(CFD_ERR_BAD_ARG, "the WENO path replaces the MUSCL reconstruction (muscl = 0 with weno = 1)");
  if (cfg->weno && cfg->precision != CFD_PREC_FP64) return fail(CFD_ERR_BAD_ARG, "the WENO path is FP64");
  if ((diss == CFD_DISS_AUSM || diss == CFD_DISS_HLLC) && cfg->is_second_order && !cfg->muscl)
    return fail(CFD_ERR_BAD_ARG, "second-order AUSM / HLLC use the gradient-MUSCL form (muscl = 1)");
  if (diss == CFD_DISS_LLF && cfg->is_second_order)
    return fail(CFD_ERR_BAD_ARG, "LLF_2O reads uninitialised state in the reference (src/LLF.cpp:101); not supported");
  if (cfg->limiter < 0 || cfg->limiter > 4) return fail(CFD_ERR_BAD_ARG, "bad limiter");
  if (!(cfg->entropy_fix_linear >= 0.0) || !std::isfinite(cfg->entropy_fix_linear))
    return fail(CFD_ERR_BAD_ARG, "entropy_fix_linear must be a finite value >= 0");
  if (!(cfg->shock_fix >= 0.0) || !std::isfinite(cfg->shock_fix))
    return fail(CFD_ERR_BAD_ARG, "shock_fix must be a finite value >= 0");
  if (cfg->reorder < 0 || cfg->reorder > 4) return fail(CFD_ERR_BAD_ARG, "reorder must be 0, 1, 2, 3 or 4");
  if (cfg->inlet_bc < 0 || cfg->inlet_bc > CFD_INLET_FARFIELD || cfg->exit_bc < 0 || cfg->exit_bc > CFD_EXIT_FIXED_P_REF)
    return fail(CFD_ERR_BAD_ARG, "bad boundary-condition kind");
  if (cfg->precision != CFD_PREC_FP64 && !(cfg->precision == CFD_PREC_FP32_FLUX && cfg->muscl && cfg->is_second_order))
    return fail(CFD_ERR_BAD_ARG, "the FP32-flux form is available for the gradient-MUSCL scheme only");

  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(CFD_ERR_NO_DEVICE, "no CUDA device");
  if (cfg->device < 0 || cfg->device >= ndev) return fail(CFD_ERR_BAD_ARG, "bad device ordinal");
  CUDA_TRY(cudaSetDevice(cfg->device));

  cfd_ctx *ctx = new cfd_ctx;
  ctx->cfg = *cfg;
  ctx->NP = NP;
  ctx->NG = NG;
  ctx->NT = NT;
  ctx->NB = NB;
  auto bail = [&](cfd_status s) {
    cfd_destroy(ctx);
    return s;
  };
  if (cfg->stream) {
    ctx->stream = static_cast<cudaStream_t>(cfg->stream);
  } else {
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess)
      return bail(fail(CFD_ERR_CUDA, "stream creation failed"));
    ctx->own_stream = true;
  }
  if (cudaMallocHost(reinterpret_cast<void **>(&ctx->h_ctl), sizeof(double) * CTL_SIZE) != cudaSuccess)
    return bail(fail(CFD_ERR_CUDA, "pinned allocation failed"));

  // Renumbering (reverse Cuthill-McKee over physical cells; ghosts keep their ids).
  BlockOrder blk;
  if (cfg->reorder == 4) {
    std::string why;
    if (!structured_block(NP, d->n_faces, d->neighbours, blk, why))
      return bail(fail(CFD_ERR_MESH, "reorder 4 needs a single structured block of quads: " + why));
    ctx->perm = blk.cell;
  } else if (cfg->reorder == 3 && d->center_vectors)
    rcb_patches(NP, d->n_faces, d->neighbours, d->center_vectors, kPatchCells, ctx->perm, ctx->patch_starts);
  else if (cfg->reorder == 2) ctx->perm = patch_from_arrays(NP, d->n_faces, d->neighbours, 128);
  else if (cfg->reorder) ctx->perm = rcm_from_arrays(NP, d->n_faces, d->neighbours);
  else {
    ctx->perm.resize(NP);
    for (int i = 0; i < NP; i++) ctx->perm[i] = i;
  }
  ctx->inv.assign(NP, 0);
  for (int i = 0; i < NP; i++) ctx->inv[ctx->perm[i]] = i;

  // Face-major SoA geometry in device order, plus the limiter stencil of
  // Second_Order_Limiter (src/Limiters.cpp:136-191) resolved once on the host.
  std::vector<int> nf(NP), nbr(4 * (size_t)NP, 0), n2(4 * (size_t)NP, 0);
  std::vector<double> nx(4 * (size_t)NP, 0.0), ny(4 * (size_t)NP, 0.0), dl(4 * (size_t)NP, 0.0);
  std::vector<double> d1l(4 * (size_t)NP, 1.0), d2l(4 * (size_t)NP, 1.0), area(NP), inva(NP);
  std::vector<double> cvx(4 * (size_t)NP, 0.0), cvy(4 * (size_t)NP, 0.0);
  if (cfg->muscl && cfg->is_second_order && !d->center_vectors)
    return bail(fail(CFD_ERR_BAD_ARG, "gradient MUSCL needs centre vectors"));
  std::vector<uint8_t> degen(NP, 0);
  const double *ccd = d->center_distances;
  for (int i = 0; i < NP; i++) {
    const int r = ctx->perm[i];
    const int nfr = d->n_faces[r];
    nf[i] = nfr;
    area[i] = d->area[r];
    inva[i] = d->inv_area[r];
    for (int f = 0; f < nfr; f++) {
      const size_t idx = (size_t)f * NP + i;
      const int N = d->neighbours[4 * r + f];
      nbr[idx] = dev_of(ctx, N);
      const double fx = d->face_normals[8 * r + 2 * f], fy = d->face_normals[8 * r + 2 * f + 1];
      nx[idx] = fx;
      ny[idx] = fy;
      dl[idx] = d->face_lengths[4 * r + f];
      if (std::sqrt(fx * fx + fy * fy) < 1e-12) degen[i] |= static_cast<uint8_t>(1u << f);
      if (d->center_vectors) {
        cvx[idx] = d->center_vectors[8 * r + 2 * f];
        cvy[idx] = d->center_vectors[8 * r + 2 * f + 1];
      }
      if (ccd) {
        int N2;
        double d1, d2;
        if (nfr != 4) {
          d1 = ccd[4 * r + f];
          if (d1 <= 0.0) d1 = 1.0;
          N2 = N;
          d2 = d1;
        } else if (f == 0 || f == 1) {
          d1 = ccd[4 * r + f];
          N2 = (N >= NP) ? N : d->neighbours[4 * N + f];
          d2 = (N >= NP) ? d1 : ccd[4 * N + f];
        } else {
          const int o = f - 2;
          d1 = ccd[4 * r + f];
          N2 = d->neighbours[4 * r + o];
          d2 = ccd[4 * r + o];
        }
        n2[idx] = dev_of(ctx, N2);
        d1l[idx] = d1;
        d2l[idx] = d2;
      }
    }
  }
  // Unique faces of the face-based (gradient MUSCL) form, numbered in reference order: a face
  // belongs to the lower-numbered of its two cells, a boundary face to its physical cell; its
  // geometry is the owner's.  Faces are stored sorted by owner in device order.
  std::vector<int> fo, fn, cface;
  std::vector<double> fnx, fny, fdl, fdx, fdy;
  if (cfg->muscl && cfg->is_second_order) {
    std::vector<int> ref_owner, ref_face;
    std::vector<int> slot_face(4 * (size_t)NP, 0);  // reference cell-major: face id or -(id+1)
    for (int r = 0; r < NP; r++)
      for (int f = 0; f < d->n_faces[r]; f++) {
        const int N = d->neighbours[4 * r + f];
        if (N < NP && N < r) continue;
        const int id = static_cast<int>(ref_owner.size());
        ref_owner.push_back(r);
        ref_face.push_back(f);
        slot_face[4 * r + f] = id;
        if (N < NP) {
          int g = -1;
          for (int k = 0; k < d->n_faces[N]; k++)
            if (d->neighbours[4 * N + k] == r) g = k;
          if (g < 0) return bail(fail(CFD_ERR_MESH, "non-conforming face between cells " + std::to_string(r) + " and " +
                                                        std::to_string(N)));
          slot_face[4 * N + g] = -(id + 1);
        }
      }
    const int NF = static_cast<int>(ref_owner.size());
    std::vector<int> order(NF);
    for (int i = 0; i < NF; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return ctx->inv[ref_owner[a]] < ctx->inv[ref_owner[b]]; });
    std::vector<int> pos(NF);
    for (int i = 0; i < NF; i++) pos[order[i]] = i;
    fo.resize(NF);
    fn.resize(NF);
    fnx.resize(NF);
    fny.resize(NF);
    fdl.resize(NF);
    fdx.resize(NF);
    fdy.resize(NF);
    for (int i = 0; i < NF; i++) {
      const int id = order[i], r = ref_owner[id], f = ref_face[id];
      fo[i] = ctx->inv[r];
      fn[i] = dev_of(ctx, d->neighbours[4 * r + f]);
      fnx[i] = d->face_normals[8 * r + 2 * f];
      fny[i] = d->face_normals[8 * r + 2 * f + 1];
      fdl[i] = d->face_lengths[4 * r + f];
      fdx[i] = d->center_vectors[8 * r + 2 * f];
      fdy[i] = d->center_vectors[8 * r + 2 * f + 1];
    }
    cface.assign(4 * (size_t)NP, 0);
    for (int i = 0; i < NP; i++) {
      const int r = ctx->perm[i];
      for (int f = 0; f < d->n_faces[r]; f++) {
        const int e = slot_face[4 * r + f];
        cface[(size_t)f * NP + i] = e >= 0 ? pos[e] : -(pos[-e - 1] + 1);
      }
    }
  }
  // Tile tables (reorder 4, face-based forms): per cell its slot rotation and the faces it owns,
  // the two structured face families with their unique-face values, and the ghost rows beside the
  // block's rim.  The form is offered only when every slot normal and length of a cell equals its
  // face's owner-side values (negated normal on the non-owner side) bit for bit, which is what the
  // kernel relies on when it forms the gradients from the face values.
  std::vector<int> tgW, tgE, tgS, tgN;
  std::vector<unsigned char> tcode, two, tso;
  std::vector<double4> tfw, tfs;
  std::vector<double> twdy, tsdy;
  bool tile_tables = false;
  if (cfg->reorder == 4 && !fo.empty()) {
    const int ni = blk.ni, nj = blk.nj;
    bool ok = true;
    tcode.assign(NP, 0);
    tfw.assign((size_t)(ni + 1) * nj, make_double4(0, 0, 0, 0));
    twdy.assign((size_t)(ni + 1) * nj, 0.0);
    two.assign((size_t)(ni + 1) * nj, 0);
    tfs.assign((size_t)ni * (nj + 1), make_double4(0, 0, 0, 0));
    tsdy.assign((size_t)ni * (nj + 1), 0.0);
    tso.assign((size_t)ni * (nj + 1), 0);
    tgW.assign(nj, 0);
    tgE.assign(nj, 0);
    tgS.assign(ni, 0);
    tgN.assign(ni, 0);
    // Face of slot s of device cell i: its id, whether the cell owns it, and the exactness check.
    auto face_of = [&](int i, int s, int &id) {
      const int e = cface[(size_t)s * NP + i];
      id = e >= 0 ? e : -e - 1;
      const size_t idx = (size_t)s * NP + i;
      const bool own = e >= 0;
      if (!(nx[idx] == (own ? fnx[id] : -fnx[id]) && ny[idx] == (own ? fny[id] : -fny[id]) && dl[idx] == fdl[id]))
        ok = false;
      return own;
    };
    for (int j = 0; j < nj && ok; j++)
      for (int i = 0; i < ni && ok; i++) {
        const int c = j * ni + i, r = ctx->perm[c];
        const int sE = blk.sE[r], sN = blk.sN[r], sW = (sE + 2) & 3, sS = (sN + 2) & 3;
        // Position p (E, N, W, S; E, S, W, N when lh) is slot (sE + p) & 3.
        unsigned char code = static_cast<unsigned char>((4 - sE) & 3);
        for (int p = 0; p < 4; p++) {
          int id;
          if (face_of(c, (sE + p) & 3, id)) code |= static_cast<unsigned char>(1u << (2 + p));
        }
        tcode[c] = code;
        int id;
        const size_t wi = (size_t)j * (ni + 1) + i;
        two[wi] = face_of(c, sW, id) ? 1 : 0;
        tfw[wi] = make_double4(fnx[id], fny[id], fdl[id], fdx[id]);
        twdy[wi] = fdy[id];
        if (i == ni - 1) {
          if (!face_of(c, sE, id)) ok = false;  // a boundary face belongs to its cell
          tfw[wi + 1] = make_double4(fnx[id], fny[id], fdl[id], fdx[id]);
          twdy[wi + 1] = fdy[id];
          two[wi + 1] = 0;
        }
        const size_t si = (size_t)j * ni + i;
        tso[si] = face_of(c, sS, id) ? 1 : 0;
        tfs[si] = make_double4(fnx[id], fny[id], fdl[id], fdx[id]);
        tsdy[si] = fdy[id];
        if (j == nj - 1) {
          if (!face_of(c, sN, id)) ok = false;
          tfs[si + ni] = make_double4(fnx[id], fny[id], fdl[id], fdx[id]);
          tsdy[si + ni] = fdy[id];
          tso[si + ni] = 0;
        }
        if (i == 0) tgW[j] = nbr[(size_t)sW * NP + c];
        if (i == ni - 1) tgE[j] = nbr[(size_t)sE * NP + c];
        if (j == 0) tgS[i] = nbr[(size_t)sS * NP + c];
        if (j == nj - 1) tgN[i] = nbr[(size_t)sN * NP + c];
      }
    tile_tables = ok;
  }
  // Patch tables of the one-kernel stage form (reorder 3): per patch its halo cells and the faces
  // touching its cells, each with the shared-memory rows of its two cells and the face slots they
  // fill.  Any inconsistency leaves the patch form off (the three-kernel form is always there).
  std::vector<int2> patches;
  std::vector<int> phptr(1, 0), phcell, pfptr(1, 0);
  std::vector<PatchFace> pface;
  int patch_rows = 0;
  if (!ctx->patch_starts.empty() && !fo.empty()) {
    const int npatch = static_cast<int>(ctx->patch_starts.size());
    std::vector<int> seen(NP, -1), loc(NP, 0);
    bool ok = true;
    auto slot_of = [&](int cell, int code) {
      for (int g = 0; g < nf[cell]; g++)
        if (cface[(size_t)g * NP + cell] == code) return g;
      return -1;
    };
    for (int b = 0; b < npatch && ok; b++) {
      const int c0 = ctx->patch_starts[b], c1 = b + 1 < npatch ? ctx->patch_starts[b + 1] : NP, P = c1 - c0;
      auto own = [&](int x) { return x >= c0 && x < c1; };
      if (P <= 0 || P > kPatchCells) {
        ok = false;
        break;
      }
      int H = 0;
      for (int c = c0; c < c1; c++)
        for (int f = 0; f < nf[c]; f++) {
          const int N = nbr[(size_t)f * NP + c];
          if (N < 0 || N >= NP || own(N) || seen[N] == b) continue;
          seen[N] = b;
          loc[N] = P + H++;
          phcell.push_back(N);
        }
      const int rows = P + H;
      if (rows >= 0xFFFF) {
        ok = false;
        break;
      }
      auto pack = [](int lo, int hi) { return static_cast<int>(static_cast<unsigned>(lo) | (static_cast<unsigned>(hi) << 16)); };
      for (int c = c0; c < c1 && ok; c++)
        for (int f = 0; f < nf[c]; f++) {
          const int e = cface[(size_t)f * NP + c];
          const int l = c - c0;
          if (e >= 0) {
            const int N = fn[e];
            int ln, sn = 0xFF;
            if (N >= NP) ln = 0xFFFF;
            else if (own(N)) {
              ln = N - c0;
              sn = slot_of(N, -(e + 1));
            } else ln = seen[N] == b ? loc[N] : -1;
            if (ln < 0 || sn < 0 || fo[e] != c || N >= NT) ok = false;
            pface.push_back({N, pack(l, ln), f | (sn << 8), e, fnx[e], fny[e], fdl[e], fdx[e], fdy[e], 0.0});
          } else {
            const int i = -e - 1, o = fo[i];
            if (own(o)) continue;  // listed from its owner's side
            if (o < 0 || o >= NP || seen[o] != b || fn[i] != c) ok = false;
            pface.push_back({c, pack(ok ? loc[o] : 0, l), 0xFF | (f << 8), i, fnx[i], fny[i], fdl[i], fdx[i], fdy[i], 0.0});
          }
        }
      patches.push_back(make_int2(c0, P));
      phptr.push_back(static_cast<int>(phcell.size()));
      pfptr.push_back(static_cast<int>(pface.size()));
      patch_rows = std::max(patch_rows, rows);
    }
    if (!ok) {
      patches.clear();
      phcell.clear();
      pface.clear();
      phptr.assign(1, 0);
      pfptr.assign(1, 0);
      patch_rows = 0;
    }
  }
  std::vector<int4> bnd(NB);
  for (int e = 0; e < NB; e++) {
    const int *b = d->boundary + 4 * e;
    bnd[e] = make_int4(b[0], dev_of(ctx, b[1]), b[2], b[3]);
  }
  // A ghost row is private when it has exactly one boundary entry and only its owner cell lists it
  // as a neighbour; then the owner's thread may apply that entry's boundary condition itself.
  {
    std::vector<int> owner(NT > NP ? NT - NP : 1, -1);
    bool priv = true;
    for (int e = 0; e < NB && priv; e++) {
      const int g = bnd[e].w - NP;
      if (owner[g] != -1) priv = false;
      owner[g] = bnd[e].y;
    }
    for (int c = 0; c < NP && priv; c++)
      for (int f = 0; f < nf[c]; f++) {
        const int N = nbr[(size_t)f * NP + c];
        if (N >= NP && owner[N - NP] != c) priv = false;
      }
    ctx->ghost_private = priv;
  }
  // Boundary entries grouped by (device) owner cell, in entry order within a cell.
  std::vector<int> bptr(NP + 1, 0), bidx(NB > 0 ? NB : 1, 0);
  for (int e = 0; e < NB; e++) bptr[bnd[e].y + 1]++;
  for (int i = 0; i < NP; i++) bptr[i + 1] += bptr[i];
  {
    std::vector<int> fill(bptr.begin(), bptr.end() - 1);
    for (int e = 0; e < NB; e++) bidx[fill[bnd[e].y]++] = e;
  }

  DevMesh &m = ctx->dm;
  m.NP = NP;
  m.NT = NT;
  m.NB = NB;
  cfd_status s;
  if ((s = ctx_upload(ctx, const_cast<int **>(&m.nf), nf)) != CFD_OK) return bail(s);
  if ((s = ctx_upload(ctx, const_cast<int **>(&m.nbr), nbr)) != CFD_OK) return bail(s);
  {
    std::vector<int4> n4(NP);
    for (int i = 0; i < NP; i++)
      n4[i] = make_int4(nbr[i], nbr[(size_t)NP + i], nbr[2 * (size_t)NP + i], nbr[3 * (size_t)NP + i]);
    if ((s = ctx_upload(ctx, const_cast<int4 **>(&m.nbr4), n4)) != CFD_OK) return bail(s);
  }
  if ((s = ctx_upload(ctx, const_cast<double **>(&m.nx), nx)) != CFD_OK) return bail(s);
  if ((s = ctx_upload(ctx, const_cast<double **>(&m.ny), ny)) != CFD_OK) return bail(s);
  if ((s = ctx_upload(ctx, const_cast<double **>(&m.dl), dl)) != CFD_OK) return bail(s);
  if ((s = ctx_upload(ctx, const_cast<double **>(&m.area), area)) != CFD_OK) return bail(s);
  if ((s = ctx_upload(ctx, const_cast<double **>(&m.inv_area), inva)) != CFD_OK) return bail(s);
  if ((s = ctx_upload(ctx, const_cast<int **>(&m.n2), n2)) != CFD_OK) return bail(s);
  if ((s = ctx_upload(ctx, const_cast<double **>(&m.d1l), d1l)) != CFD_OK) return bail(s);
  if ((s = ctx_upload(ctx, const_cast<double **>(&m.d2l), d2l)) != CFD_OK) return bail(s);
  if ((s = ctx_upload(ctx, const_cast<uint8_t **>(&m.degen), degen)) != CFD_OK) return bail(s);
  if ((s = ctx_upload(ctx, const_cast<double **>(&m.cvx), cvx)) != CFD_OK) return bail(s);
  if ((s = ctx_upload(ctx, const_cast<double **>(&m.cvy), cvy)) != CFD_OK) return bail(s);
  if ((s = ctx_upload(ctx, const_cast<int4 **>(&m.bnd), bnd)) != CFD_OK) return bail(s);
  if ((s = ctx_upload(ctx, const_cast<int **>(&m.bptr), bptr)) != CFD_OK) return bail(s);
  if ((s = ctx_upload(ctx, const_cast<int **>(&m.bidx), bidx)) != CFD_OK) return bail(s);
  m.NF = static_cast<int>(fo.size());
  if (m.NF > 0) {
    if ((s = ctx_upload(ctx, const_cast<int **>(&m.fo), fo)) != CFD_OK) return bail(s);
    if ((s = ctx_upload(ctx, const_cast<int **>(&m.fn), fn)) != CFD_OK) return bail(s);
    if ((s = ctx_upload(ctx, const_cast<double **>(&m.fnx), fnx)) != CFD_OK) return bail(s);
    if ((s = ctx_upload(ctx, const_cast<double **>(&m.fny), fny)) != CFD_OK) return bail(s);
    if ((s = ctx_upload(ctx, const_cast<double **>(&m.fdl), fdl)) != CFD_OK) return bail(s);
    if ((s = ctx_upload(ctx, const_cast<double **>(&m.fdx), fdx)) != CFD_OK) return bail(s);
    if ((s = ctx_upload(ctx, const_cast<double **>(&m.fdy), fdy)) != CFD_OK) return bail(s);
    {
      std::vector<int2> on(fo.size());
      std::vector<double4> g4(fo.size());
      for (size_t i = 0; i < fo.size(); i++) {
        on[i] = make_int2(fo[i], fn[i]);
        g4[i] = make_double4(fnx[i], fny[i], fdl[i], fdx[i]);
      }
      if ((s = ctx_upload(ctx, const_cast<int2 **>(&m.fon), on)) != CFD_OK) return bail(s);
      if ((s = ctx_upload(ctx, const_cast<double4 **>(&m.fg4), g4)) != CFD_OK) return bail(s);
    }
    if ((s = ctx_upload(ctx, const_cast<int **>(&m.cface), cface)) != CFD_OK) return bail(s);
    std::vector<int4> c4(NP);
    for (int i = 0; i < NP; i++)
      c4[i] = make_int4(cface[i], cface[(size_t)NP + i], cface[2 * (size_t)NP + i], cface[3 * (size_t)NP + i]);
    if ((s = ctx_upload(ctx, const_cast<int4 **>(&m.cface4), c4)) != CFD_OK) return bail(s);
  }

  m.wave_blocks = gather_stage_wave_blocks();
  if (tile_tables && tile_prepare()) {
    TileMesh &tm = ctx->tm;
    tm.ni = blk.ni;
    tm.nj = blk.nj;
    tm.lh = blk.lh;
    tm.tiles_i = (blk.ni + kTileCellsX - 1) / kTileCellsX;
    tm.tiles_j = (blk.nj + kTileCellsY - 1) / kTileCellsY;
    if ((s = ctx_upload(ctx, const_cast<int **>(&tm.gW), tgW)) != CFD_OK) return bail(s);
    if ((s = ctx_upload(ctx, const_cast<int **>(&tm.gE), tgE)) != CFD_OK) return bail(s);
    if ((s = ctx_upload(ctx, const_cast<int **>(&tm.gS), tgS)) != CFD_OK) return bail(s);
    if ((s = ctx_upload(ctx, const_cast<int **>(&tm.gN), tgN)) != CFD_OK) return bail(s);
    if ((s = ctx_upload(ctx, const_cast<unsigned char **>(&tm.code), tcode)) != CFD_OK) return bail(s);
    if ((s = ctx_upload(ctx, const_cast<double4 **>(&tm.fw), tfw)) != CFD_OK) return bail(s);
    if ((s = ctx_upload(ctx, const_cast<double **>(&tm.fwdy), twdy)) != CFD_OK) return bail(s);
    if ((s = ctx_upload(ctx, const_cast<unsigned char **>(&tm.fwo), two)) != CFD_OK) return bail(s);
    if ((s = ctx_upload(ctx, const_cast<double4 **>(&tm.fs), tfs)) != CFD_OK) return bail(s);
    if ((s = ctx_upload(ctx, const_cast<double **>(&tm.fsdy), tsdy)) != CFD_OK) return bail(s);
    if ((s = ctx_upload(ctx, const_cast<unsigned char **>(&tm.fso), tso)) != CFD_OK) return bail(s);
    // 48-byte face records of the TMA form: nx, ny, dl, dx, dy, owner on the high side.
    std::vector<double> gw6(tfw.size() * 6), gs6(tfs.size() * 6);
    for (size_t f = 0; f < tfw.size(); f++) {
      const double r[6] = {tfw[f].x, tfw[f].y, tfw[f].z, tfw[f].w, twdy[f], two[f] ? 1.0 : 0.0};
      std::copy(r, r + 6, gw6.begin() + 6 * f);
    }
    for (size_t f = 0; f < tfs.size(); f++) {
      const double r[6] = {tfs[f].x, tfs[f].y, tfs[f].z, tfs[f].w, tsdy[f], tso[f] ? 1.0 : 0.0};
      std::copy(r, r + 6, gs6.begin() + 6 * f);
    }
    if ((s = ctx_upload(ctx, const_cast<double **>(&tm.gw6), gw6)) != CFD_OK) return bail(s);
    if ((s = ctx_upload(ctx, const_cast<double **>(&tm.gs6), gs6)) != CFD_OK) return bail(s);
    ctx->tile_ok = true;
  }
  if (!patches.empty()) {
    m.npatch = static_cast<int>(patches.size());
    m.patch_rows = patch_rows;
    if (!patch_prepare(m)) m.npatch = 0;
  }
  if (m.npatch > 0) {
    if ((s = ctx_upload(ctx, const_cast<int2 **>(&m.patch), patches)) != CFD_OK) return bail(s);
    if ((s = ctx_upload(ctx, const_cast<int **>(&m.phptr), phptr)) != CFD_OK) return bail(s);
    if ((s = ctx_upload(ctx, const_cast<int **>(&m.phcell), phcell)) != CFD_OK) return bail(s);
    if ((s = ctx_upload(ctx, const_cast<int **>(&m.pfptr), pfptr)) != CFD_OK) return bail(s);
    if ((s = ctx_upload(ctx, const_cast<PatchFace **>(&m.pface), pface)) != CFD_OK) return bail(s);
  }

  DevState &st = ctx->ds;
  const size_t dsz = sizeof(double);
  const int nblk = std::max(std::max(flux_block_count(NP), m.npatch), ctx->tile_ok ? ctx->tm.tiles_i * ctx->tm.tiles_j : 0);
  ctx->partial_blocks = nblk;
  if ((s = ctx_alloc(ctx, (void **)&st.U, 4 * (size_t)NT * dsz)) != CFD_OK) return bail(s);
  if ((s = ctx_alloc(ctx, (void **)&st.S, 4 * (size_t)NP * dsz)) != CFD_OK) return bail(s);
  if ((s = ctx_alloc(ctx, (void **)&st.prim, 5 * (size_t)NT * dsz)) != CFD_OK) return bail(s);
  if ((s = ctx_alloc(ctx, (void **)&st.R, 4 * (size_t)NP * dsz)) != CFD_OK) return bail(s);
  if ((s = ctx_alloc(ctx, (void **)&st.dtc, (size_t)NP * dsz)) != CFD_OK) return bail(s);
  if ((s = ctx_alloc(ctx, (void **)&st.dtk, (size_t)NP * dsz)) != CFD_OK) return bail(s);
  if ((s = ctx_alloc(ctx, (void **)&st.dU, 4 * (size_t)NP * dsz)) != CFD_OK) return bail(s);
  if (cfg->integrator == CFD_INT_RK4) {
    if ((s = ctx_alloc(ctx, (void **)&st.Racc, 4 * (size_t)NP * dsz)) != CFD_OK) return bail(s);
  }
  if (cfg->muscl) {
    if (cfg->precision == CFD_PREC_FP32_FLUX) {
      if ((s = ctx_alloc(ctx, (void **)&st.recf, 2 * (size_t)NP * sizeof(float4))) != CFD_OK) return bail(s);
    } else if ((s = ctx_alloc(ctx, (void **)&st.rec, 8 * (size_t)NP * dsz)) != CFD_OK) {
      return bail(s);
    }
    if ((s = ctx_alloc(ctx, (void **)&st.q4, ((size_t)NT + (size_t)m.NF) * sizeof(double4))) != CFD_OK) return bail(s);
    if (cudaMemset(st.q4, 0, (size_t)NT * sizeof(double4)) != cudaSuccess) return bail(fail(CFD_ERR_CUDA, "memset failed"));
    if (m.NF > 0) st.F = st.q4 + NT;
  }
  if (m.NF > 0 && !st.F) {
    if ((s = ctx_alloc(ctx, (void **)&st.F, 4 * (size_t)m.NF * dsz)) != CFD_OK) return bail(s);
  }
  if ((s = ctx_alloc(ctx, (void **)&st.ctl, CTL_SIZE * dsz)) != CFD_OK) return bail(s);
  // Face-based forms: the (rho, u, v, p) rows and the face fluxes, one allocation (rows first), are
  // kept in L2 as persisting lines: the gather writes the rows that the gradient and face kernels
  // read next, and the face kernel writes the fluxes the gather reads right after.  The device's
  // persisting set-aside is raised to hold them (up to the device maximum; never lowered; it lasts
  // as long as this process's CUDA context).  Only when the whole region fits in the largest
  // set-aside the device allows (quad meshes up to about 0.86 M cells on B200); a partial window was
  // not measured to help.
  if (m.NF > 0) {
    int maxp = 0, maxw = 0;
    size_t cur = 0;
    const size_t fb = 4 * ((size_t)m.NF + (st.q4 ? (size_t)NT : 0)) * dsz;
    if (cudaDeviceGetAttribute(&maxp, cudaDevAttrMaxPersistingL2CacheSize, cfg->device) == cudaSuccess &&
        cudaDeviceGetAttribute(&maxw, cudaDevAttrMaxAccessPolicyWindowSize, cfg->device) == cudaSuccess &&
        maxp > 0 && maxw > 0 && fb <= (size_t)maxp && fb <= (size_t)maxw &&
        cudaDeviceGetLimit(&cur, cudaLimitPersistingL2CacheSize) == cudaSuccess) {
      const size_t want = std::min<size_t>((size_t)maxp, fb);
      if (cur < want && cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want) == cudaSuccess) cur = want;
      if (cur > 0) {
        m.l2_base = st.q4 ? (void *)st.q4 : (void *)st.F;
        m.l2_bytes = std::min<size_t>(fb, (size_t)maxw);
        m.l2_hit = std::min(1.0f, (float)cur / (float)m.l2_bytes);
        ctx->l2_window = m.l2_bytes;
      }
    }
    cudaGetLastError();
  }
  for (int q = 0; q < 2 && ctx->tile_ok; q++) {
    if ((s = ctx_alloc(ctx, (void **)&ctx->qbuf[q], (size_t)NT * sizeof(double4))) != CFD_OK) return bail(s);
    if (cudaMemset(ctx->qbuf[q], 0, (size_t)NT * sizeof(double4)) != cudaSuccess)
      return bail(fail(CFD_ERR_CUDA, "memset failed"));
  }
  ctx->tile_stage = 0;
  if (ctx->tile_ok && tile_tma_prepare()) {
    double4 *bufs[3] = {ctx->ds.q4, ctx->qbuf[0], ctx->qbuf[1]};
    int bq[3], bw[3], bs[3];
    tile_tma_boxes(bq, bw, bs);
    const TileMesh &tm = ctx->tm;
    bool ok = true;
    for (int q = 0; q < 3; q++)
      ok = ok && encode_tensor_3d(&ctx->tmap_q[q], bufs[q], 4, tm.ni, tm.nj, bq);
    ok = ok && encode_tensor_3d(&ctx->tmap_gw, tm.gw6, 6, tm.ni + 1, tm.nj, bw);
    ok = ok && encode_tensor_3d(&ctx->tmap_gs, tm.gs6, 6, tm.ni, tm.nj + 1, bs);
    ctx->tile_tma_ok = ok;
  }
  for (int q = 0; q < 2 && m.npatch > 0; q++) {
    if ((s = ctx_alloc(ctx, (void **)&ctx->pbuf[q], 5 * (size_t)NT * dsz)) != CFD_OK) return bail(s);
    if (cudaMemset(ctx->pbuf[q], 0, 5 * (size_t)NT * dsz) != cudaSuccess) return bail(fail(CFD_ERR_CUDA, "memset failed"));
  }
  if ((s = ctx_alloc(ctx, (void **)&st.partial, 9 * (size_t)(nblk + kMaxGroups) * dsz)) != CFD_OK) return bail(s);
  const size_t counter_bytes = 64 + 4 * (size_t)(kMaxGroups + 1);
  if ((s = ctx_alloc(ctx, (void **)&st.counter, counter_bytes)) != CFD_OK) return bail(s);
  st.gcount = st.counter + 16;
  if ((s = ctx_alloc(ctx, (void **)&st.status, 64)) != CFD_OK) return bail(s);
  if (cudaMemset(st.U, 0, 4 * (size_t)NT * dsz) != cudaSuccess || cudaMemset(st.S, 0, 4 * (size_t)NP * dsz) != cudaSuccess ||
      cudaMemset(st.prim, 0, 5 * (size_t)NT * dsz) != cudaSuccess || cudaMemset(st.R, 0, 4 * (size_t)NP * dsz) != cudaSuccess ||
      cudaMemset(st.dtc, 0, (size_t)NP * dsz) != cudaSuccess || cudaMemset(st.dU, 0, 4 * (size_t)NP * dsz) != cudaSuccess ||
      cudaMemset(st.ctl, 0, CTL_SIZE * dsz) != cudaSuccess || cudaMemset(st.counter, 0, counter_bytes) != cudaSuccess)
    return bail(fail(CFD_ERR_CUDA, "memset failed"));
  int hs[2] = {0, INT_MAX};
  if (cudaMemcpy(st.status, hs, sizeof(hs), cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(fail(CFD_ERR_CUDA, "status init failed"));
  if ((s = ctx_upload(ctx, &ctx->d_perm, ctx->perm)) != CFD_OK) return bail(s);
  if ((s = ctx_alloc(ctx, (void **)&ctx->d_stage, 4 * (size_t)NT * dsz)) != CFD_OK) return bail(s);

  FluxParams &fp = ctx->fp;
  fp.dissipation = diss;
  fp.movers_single = cfg->movers_single_alpha ? 1 : 0;
  fp.movers_efix = cfg->movers_entropy_fix ? 1 : 0;
  fp.second_order = cfg->is_second_order;
  fp.limiter = cfg->limiter;
  fp.recon_prim = cfg->reconstruct_primitive;
  fp.muscl = cfg->muscl && cfg->is_second_order;
  fp.lanes = 1;
  fp.faces_shape = 3;
  // WENO (Is_WENO): Explicit_Method falls back to the 1O/2O residual when any cell is not a quad
  // (src/Numerical_Method.cpp:31-55); Runge_Kutta_Method keeps WENO (zero flux on those cells).
  {
    bool all_quads = true;
    for (int c = 0; c < NP; c++) all_quads = all_quads && d->n_faces[c] == 4;
    const bool explicit_form = cfg->integrator == CFD_INT_REFERENCE && !cfg->time_accurate;
    fp.weno = cfg->weno && (all_quads || !explicit_form) ? 1 : 0;
    fp.weno_char = cfg->weno_characteristic ? 1 : 0;
  }
  fp.consistent = (cfg->integrator != CFD_INT_REFERENCE) ? 1 : 0;
  fp.precision = cfg->precision;
  fp.cfl = cfg->cfl;
  fp.zeta = cfg->limiter_zeta;
  fp.zeta1 = cfg->limiter_zeta1;
  fp.eflin = cfg->entropy_fix_linear;
  fp.shock_fix = cfg->shock_fix;
  BcParams &bp = ctx->bp;
  bp.inlet_bc = cfg->inlet_bc;
  bp.exit_bc = cfg->exit_bc;
  bp.inlet_rho = cfg->inlet_rho;
  bp.inlet_p = cfg->inlet_p;
  bp.inlet_u = cfg->inlet_u;
  bp.inlet_v = cfg->inlet_v;
  bp.inlet_p0 = cfg->inlet_p0;
  bp.inlet_t0 = cfg->inlet_t0;
  bp.exit_p = cfg->exit_p;
  bp.r_gas = cfg->r_gas > 0.0 ? cfg->r_gas : 287.0;
  *out = ctx;
  return CFD_OK;
}

cfd_status cfd_set_option(cfd_ctx *ctx, const char *name, double value) {
  if (!ctx || !name) return fail(CFD_ERR_BAD_ARG, "null argument");
  std::string n(name);
  if (n == "persistent") {
    // Persistent batched form: one cooperative launch per RK stage over the work lists, at most
    // the co-resident grid and the reduction buffers' block count.
    drop_graphs(ctx);
    ctx->persistent = false;
    ctx->persist_grid = 0;
    if (value != 0.0) {
      const int g = persistent_grid(ctx->fp);
      if (g <= 0) return fail(CFD_ERR_BAD_ARG, "cooperative launches are not available on this device");
      ctx->persistent = true;
      ctx->persist_grid = std::min(g, ctx->partial_blocks);
    }
    return CFD_OK;
  }
  if (n == "persist_minb") {
    // Register budget of the persistent stage kernel (4, 6 or 8 resident blocks per SM); the
    // co-resident grid follows.
    if (value != 0.0 && value != 4.0 && value != 6.0 && value != 8.0)
      return fail(CFD_ERR_BAD_ARG, "persist_minb must be 0, 4, 6 or 8");
    drop_graphs(ctx);
    ctx->fp.persist_minb = static_cast<int>(value);
    if (ctx->persistent) {
      const int g = persistent_grid(ctx->fp);
      if (g <= 0) return fail(CFD_ERR_BAD_ARG, "cooperative launches are not available on this device");
      ctx->persist_grid = std::min(g, ctx->partial_blocks);
    }
    return CFD_OK;
  }
  if (n == "barrier_timeout_test") {
    // Test of the bounded barrier: every barrier of the persistent form waits for `value` more
    // arrivals than the grid has, so each wait runs out and the run reports CFD_ERR_TIMEOUT.
    drop_graphs(ctx);
    ctx->persist_test_arrivals = value > 0.0 ? static_cast<unsigned int>(value) : 0u;
    return CFD_OK;
  }
  if (n == "keep_delu") ctx->keep_delu = value != 0.0;
  else if (n == "use_graph") ctx->use_graph = value != 0.0;
  else if (n == "flux_minb") {
    if (value != 1.0 && value != 6.0 && value != 8.0) return fail(CFD_ERR_BAD_ARG, "flux_minb must be 1, 6 or 8");
    ctx->fp.flux_minb = static_cast<int>(value);
    drop_graphs(ctx);
  } else if (n == "flux_lanes") {
    if (value != 1.0 && value != 4.0) return fail(CFD_ERR_BAD_ARG, "flux_lanes must be 1 or 4");
    ctx->fp.lanes = static_cast<int>(value);
  }
  else if (n == "faces_shape") {
    if (value != 0.0 && value != 1.0 && value != 2.0 && value != 3.0 && value != 4.0)
      return fail(CFD_ERR_BAD_ARG, "faces_shape must be 0, 1, 2, 3 or 4");
    ctx->fp.faces_shape = static_cast<int>(value);
  }
  else if (n == "pdl") ctx->dm.pdl = value != 0.0;
  else if (n == "profile") ctx->profile = value != 0.0;
  else if (n == "fuse_gather") ctx->fuse_gather = value != 0.0;
  else if (n == "patch_stage") ctx->patch_stage = value != 0.0;
  else if (n == "tile_stage") {
    if (value != 0.0 && value != 1.0 && value != 2.0 && value != 3.0 && value != 4.0)
      return fail(CFD_ERR_BAD_ARG, "tile_stage must be 0, 1, 2, 3 or 4");
    if (value != 0.0 && !ctx->tile_ok)
      return fail(CFD_ERR_BAD_ARG, "the tile form needs reorder 4 on a structured block with the gradient-MUSCL scheme");
    if (value >= 2.0 && !ctx->tile_tma_ok)
      return fail(CFD_ERR_BAD_ARG, "the TMA tile form is not available on this device");
    ctx->tile_stage = static_cast<int>(value);
  }
  else if (n == "l2_persist") ctx->dm.l2_bytes = value != 0.0 ? ctx->l2_window : 0;
  else if (n == "tile_prefetch") ctx->tm.prefetch_ahead = value != 0.0;
  else return fail(CFD_ERR_BAD_ARG, "unknown option " + n);
  drop_graphs(ctx);
  return CFD_OK;
}

cfd_status cfd_upload_state(cfd_ctx *ctx, const double *U, int n) {
  if (!ctx || !U) return fail(CFD_ERR_BAD_ARG, "null argument");
  if (n != ctx->NP && n != ctx->NT) return fail(CFD_ERR_BAD_ARG, "n must be NP or NP+NG");
  const int NT = ctx->NT, NP = ctx->NP;
  // Rows go to a device staging buffer in reference order; a kernel gathers them into the
  // device-order planes.  With n = NP the ghost rows are filled from their owner cell first.
  CUDA_TRY(cudaMemcpyAsync(ctx->d_stage, U, 4 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  if (n == NP && ctx->NB > 0) {
    std::vector<int4> bnd(ctx->NB);
    CUDA_TRY(cudaMemcpy(bnd.data(), ctx->dm.bnd, ctx->NB * sizeof(int4), cudaMemcpyDeviceToHost));
    for (const int4 &b : bnd)
      CUDA_TRY(cudaMemcpyAsync(ctx->d_stage + 4 * (size_t)b.w, U + 4 * (size_t)ctx->perm[b.y], 4 * sizeof(double),
                               cudaMemcpyHostToDevice, ctx->stream));
  }
  ctx->launches += launch_import_aos(ctx->stream, ctx->d_stage, ctx->d_perm, NP, NT, ctx->ds.U);
  ctx->launches += launch_prim_all(ctx->stream, ctx->dm, ctx->ds);
  CUDA_TRY(cudaGetLastError());
  ctx->prim_from_S = false;
  return sync_status(ctx, nullptr);
}

cfd_status cfd_upload_state_async(cfd_ctx *ctx, const double *U, int n) {
  if (!ctx || !U) return fail(CFD_ERR_BAD_ARG, "null argument");
  if (n != ctx->NT) return fail(CFD_ERR_BAD_ARG, "the asynchronous upload takes all NP+NG rows");
  CUDA_TRY(cudaMemcpyAsync(ctx->d_stage, U, 4 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  ctx->launches += launch_import_aos(ctx->stream, ctx->d_stage, ctx->d_perm, ctx->NP, ctx->NT, ctx->ds.U);
  ctx->launches += launch_prim_all(ctx->stream, ctx->dm, ctx->ds);
  CUDA_TRY(cudaGetLastError());
  ctx->prim_from_S = false;
  return CFD_OK;
}

cfd_status cfd_download_U_async(cfd_ctx *ctx, double *U) {
  if (!ctx || !U) return fail(CFD_ERR_BAD_ARG, "null argument");
  ctx->launches += launch_export_aos(ctx->stream, ctx->ds.U, ctx->d_perm, ctx->NP, ctx->NT, ctx->NT, ctx->d_stage);
  CUDA_TRY(cudaMemcpyAsync(U, ctx->d_stage, 4 * (size_t)ctx->NT * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaGetLastError());
  return CFD_OK;
}

// Conserved rows U_Cells [(NP+NG)*4] in reference order, gathered on the device.
cfd_status cfd_download_U(cfd_ctx *ctx, double *U) {
  if (!ctx || !U) return fail(CFD_ERR_BAD_ARG, "null argument");
  ctx->launches += launch_export_aos(ctx->stream, ctx->ds.U, ctx->d_perm, ctx->NP, ctx->NT, ctx->NT, ctx->d_stage);
  CUDA_TRY(cudaMemcpyAsync(U, ctx->d_stage, 4 * (size_t)ctx->NT * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return CFD_OK;
}

// Persistent form: one CUDA graph per RK stage (each holds the stage's boundary-condition launch,
// if any, and its cooperative launch), replayed stage after stage.  A capture the driver rejects
// leaves the form on plain launches.
static cfd_status enqueue_steps_persistent(cfd_ctx *ctx, int n_steps) {
  const StagePlan p = stage_plan(ctx->cfg, ctx->fp.consistent);
  if (ctx->use_graph && !ctx->profile && ctx->stage_graphs_ok && ctx->n_stage_graphs == 0) {
    bool gw = false;
    for (int k = 0; k < p.n && ctx->stage_graphs_ok; k++) {
      cudaGraph_t g;
      CUDA_TRY(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
      ctx->stage_graph_launches[k] = enqueue_stage(ctx, k, true, gw);
      cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
      if (e == cudaSuccess) {
        e = cudaGraphInstantiate(&ctx->stage_graph[k], g, 0);
        cudaGraphDestroy(g);
      }
      if (e != cudaSuccess) {
        cudaGetLastError();
        ctx->stage_graphs_ok = false;
      }
    }
    if (ctx->stage_graphs_ok) ctx->n_stage_graphs = p.n;
    else drop_graphs(ctx);
  }
  for (int i = 0; i < n_steps; i++) {
    if (ctx->n_stage_graphs == p.n) {
      for (int k = 0; k < p.n; k++) {
        CUDA_TRY(cudaGraphLaunch(ctx->stage_graph[k], ctx->stream));
        ctx->launches += ctx->stage_graph_launches[k];
      }
    } else {
      ctx->launches += enqueue_step(ctx, true);
    }
  }
  CUDA_TRY(cudaGetLastError());
  ctx->prim_from_S = false;
  return CFD_OK;
}

static cfd_status enqueue_steps(cfd_ctx *ctx, int n_steps) {
  if (ctx->persistent && ctx->persist_grid > 0 && ctx->dm.NF > 0) return enqueue_steps_persistent(ctx, n_steps);
  if (ctx->use_graph && !ctx->profile && n_steps > 1) {
    if (!ctx->graph) {
      cudaGraph_t g;
      CUDA_TRY(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
      ctx->graph_launches = enqueue_step(ctx, true);
      cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
      if (e != cudaSuccess) return fail(CFD_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
      e = cudaGraphInstantiate(&ctx->graph, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return fail(CFD_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    }
    for (int i = 0; i < n_steps; i++) {
      CUDA_TRY(cudaGraphLaunch(ctx->graph, ctx->stream));
      ctx->launches += ctx->graph_launches;
    }
  } else {
    for (int i = 0; i < n_steps; i++) ctx->launches += enqueue_step(ctx, true);
  }
  CUDA_TRY(cudaGetLastError());
  ctx->prim_from_S = false;
  return CFD_OK;
}

cfd_status cfd_step(cfd_ctx *ctx, int n_steps, double t_end, cfd_step_info *info) {
  if (!ctx || n_steps < 0) return fail(CFD_ERR_BAD_ARG, "bad argument");
  ctx->launches += launch_set_ctl(ctx->stream, ctx->ds, CTL_TEND, t_end);
  ctx->launches += launch_set_ctl(ctx->stream, ctx->ds, CTL_DONE, 0.0);
  CUDA_TRY(cudaGetLastError());
  if (t_end > 0.0) {
    // Steps past t_end are no-ops on the device; check the done flag between chunks so that a
    // large n_steps does not queue work that will be skipped.
    const int chunk = 64;
    for (int done = 0; done < n_steps; done += chunk) {
      cfd_status s = enqueue_steps(ctx, std::min(chunk, n_steps - done));
      if (s != CFD_OK) return s;
      s = sync_status(ctx, info);
      if (s != CFD_OK) return s;
      if (ctx->h_ctl[CTL_DONE] != 0.0) break;
    }
    return sync_status(ctx, info);
  }
  cfd_status s = enqueue_steps(ctx, n_steps);
  if (s != CFD_OK) return s;
  return sync_status(ctx, info);
}

// Enqueues n pseudo-steps without waiting (benchmark helper); cfd_sync collects the status.
cfd_status cfd_step_async(cfd_ctx *ctx, int n_steps) {
  if (!ctx || n_steps < 0) return fail(CFD_ERR_BAD_ARG, "bad argument");
  return enqueue_steps(ctx, n_steps);
}

cfd_status cfd_sync(cfd_ctx *ctx, cfd_step_info *info) {
  if (!ctx) return fail(CFD_ERR_BAD_ARG, "null context");
  return sync_status(ctx, info);
}

cfd_status cfd_apply_boundary_conditions(cfd_ctx *ctx) {
  if (!ctx) return fail(CFD_ERR_BAD_ARG, "null context");
  ctx->launches += launch_bc(ctx->stream, ctx->dm, ctx->ds, ctx->bp, 0, 0);
  CUDA_TRY(cudaGetLastError());
  return sync_status(ctx, nullptr);
}

cfd_status cfd_evaluate_net_flux(cfd_ctx *ctx) {
  if (!ctx) return fail(CFD_ERR_BAD_ARG, "null context");
  ctx->launches += launch_flux(ctx->stream, ctx->dm, ctx->ds, ctx->fp, 0);
  CUDA_TRY(cudaGetLastError());
  return sync_status(ctx, nullptr);
}

// Lax_Fedrichs, src/Numerical_Method.cpp:459-481.  The wavefront schedule (reference order: a
// cell's level is one more than the highest level of its physical neighbours with a lower
// reference index) is built at the first call from the device's face table.
cfd_status cfd_lax_friedrichs(cfd_ctx *ctx) {
  if (!ctx) return fail(CFD_ERR_BAD_ARG, "null context");
  const int NP = ctx->NP;
  if (!ctx->d_lf_cells) {
    std::vector<int> nf(NP), nbr(4 * (size_t)NP);
    CUDA_TRY(cudaMemcpy(nf.data(), ctx->dm.nf, NP * sizeof(int), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(nbr.data(), ctx->dm.nbr, 4 * (size_t)NP * sizeof(int), cudaMemcpyDeviceToHost));
    for (int i = 0; i < NP; i++)
      if (nf[i] != 4) return fail(CFD_ERR_MESH, "Lax_Fedrichs reads four neighbours per cell: quad meshes only");
    std::vector<int> level(NP, 0);
    int nlev = 0;
    for (int r = 0; r < NP; r++) {
      const int i = ctx->inv[r];
      int l = 0;
      for (int f = 0; f < 4; f++) {
        const int n = nbr[(size_t)f * NP + i];
        if (n < NP && ctx->perm[n] < r) l = std::max(l, level[ctx->perm[n]] + 1);
      }
      level[r] = l;
      nlev = std::max(nlev, l + 1);
    }
    std::vector<int> start(nlev + 1, 0), cells(NP);
    for (int r = 0; r < NP; r++) start[level[r] + 1]++;
    for (int l = 0; l < nlev; l++) start[l + 1] += start[l];
    std::vector<int> fill(start.begin(), start.end() - 1);
    for (int r = 0; r < NP; r++) cells[fill[level[r]]++] = ctx->inv[r];
    int *d = nullptr;
    cfd_status s = ctx_alloc(ctx, (void **)&d, NP * sizeof(int));
    if (s != CFD_OK) return s;
    CUDA_TRY(cudaMemcpy(d, cells.data(), NP * sizeof(int), cudaMemcpyHostToDevice));
    ctx->d_lf_cells = d;
    ctx->lf_level_start = start;
  }
  ctx->launches += launch_lax_friedrichs(ctx->stream, ctx->dm, ctx->ds, ctx->d_lf_cells, ctx->lf_level_start);
  CUDA_TRY(cudaGetLastError());
  return sync_status(ctx, nullptr);
}

cfd_status cfd_explicit_method(cfd_ctx *ctx) {
  if (!ctx) return fail(CFD_ERR_BAD_ARG, "null context");
  ctx->launches += launch_flux(ctx->stream, ctx->dm, ctx->ds, ctx->fp, 0);
  cfd_status s = sync_status(ctx, nullptr);
  if (s != CFD_OK) return s;
  if (!(ctx->h_ctl[CTL_DTMIN] > 0.0)) return fail(CFD_ERR_DT_NONPOSITIVE, "Min_dt is not positive");
  ctx->launches += launch_stage(ctx->stream, ctx->dm, ctx->ds, 0, 0, 0, 1);
  CUDA_TRY(cudaGetLastError());
  return sync_status(ctx, nullptr);
}

cfd_status cfd_runge_kutta_method(cfd_ctx *ctx) {
  if (!ctx) return fail(CFD_ERR_BAD_ARG, "null context");
  const cfd_config &c = ctx->cfg;
  StagePlan p = stage_plan(c, ctx->fp.consistent);
  if (p.kind0 == 0) p = {3, 1, ctx->fp.consistent, 0};  // the reference's RK3 on an explicit config
  for (int k = 0; k < p.n; k++) {
    if (k > 0) ctx->launches += launch_bc(ctx->stream, ctx->dm, ctx->ds, ctx->bp, p.src_S, 1);
    ctx->launches += launch_flux(ctx->stream, ctx->dm, ctx->ds, ctx->fp, k > 0);
    ctx->launches += launch_stage(ctx->stream, ctx->dm, ctx->ds, p.kind0 + k, stage_lts(p, c, k), 0, 1);
  }
  CUDA_TRY(cudaGetLastError());
  ctx->prim_from_S = true;
  return sync_status(ctx, nullptr);
}

cfd_status cfd_estimate_error(cfd_ctx *ctx, double error[4]) {
  if (!ctx) return fail(CFD_ERR_BAD_ARG, "null context");
  ctx->launches += launch_error(ctx->stream, ctx->dm, ctx->ds);
  CUDA_TRY(cudaGetLastError());
  cfd_status s = sync_status(ctx, nullptr);
  if (s == CFD_OK && error)
    for (int k = 0; k < 4; k++) error[k] = ctx->h_ctl[CTL_ERR + k];
  return s;
}

// Set_DelU (src/Basic_Functions.cpp:9-18): the caller's increments [NP][4] in reference order
// replace the device's dU, so that the next cfd_update applies U += dU.
cfd_status cfd_set_delu(cfd_ctx *ctx, const double *dU) {
  if (!ctx || !dU) return fail(CFD_ERR_BAD_ARG, "null argument");
  const int NP = ctx->NP;
  std::vector<double> h(4 * (size_t)NP);
  for (int i = 0; i < NP; i++) {
    const int r = ctx->perm[i];
    for (int k = 0; k < 4; k++) h[k * (size_t)NP + i] = dU[4 * (size_t)r + k];
  }
  CUDA_TRY(cudaMemcpyAsync(ctx->ds.dU, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  return sync_status(ctx, nullptr);
}

cfd_status cfd_update(cfd_ctx *ctx) {
  if (!ctx) return fail(CFD_ERR_BAD_ARG, "null context");
  const int direct = ctx->cfg.integrator == CFD_INT_RK3_GPU_REF || ctx->cfg.integrator == CFD_INT_RK4_GPU_REF;
  ctx->launches += launch_update(ctx->stream, ctx->dm, ctx->ds, direct);
  CUDA_TRY(cudaGetLastError());
  ctx->prim_from_S = false;
  return sync_status(ctx, nullptr);
}

// Write_Solution type 1 (src/output_files.cpp:492-556): the header integers, No_Physical_Cells,
// iterations, then per cell its id, del_t, rho, p, T, u, v, M and p0 with the reference's stream
// formatting (default precision, its separators) in reference cell order.
cfd_status cfd_write_solution(cfd_ctx *ctx, const char *path, const int *header, int n_header) {
  if (!ctx || !path || n_header < 0 || (n_header > 0 && !header)) return fail(CFD_ERR_BAD_ARG, "bad argument");
  const int NP = ctx->NP, NT = ctx->NT;
  std::vector<double> P(11 * (size_t)NT), dt(NP);
  cfd_status s = cfd_download(ctx, nullptr, P.data(), dt.data(), nullptr, nullptr);
  if (s != CFD_OK) return s;
  if ((s = sync_status(ctx, nullptr)) != CFD_OK) return s;
  std::ofstream out(path);
  if (!out.is_open()) return fail(CFD_ERR_IO, std::string("cannot write ") + path);
  for (int k = 0; k < n_header; k++) out << header[k] << (k + 1 < n_header ? "\t" : "");
  out << std::endl;
  out << NP << std::endl;
  out << static_cast<int>(ctx->h_ctl[CTL_ITER]) << std::endl;
  for (int c = 0; c < NP; c++) {
    const double *q = P.data() + 11 * (size_t)c;
    out << c << "\t\t" << dt[c] << "\t" << q[0] << "\t" << q[4] << "\t" << q[3] << "\t\t\t\t" << q[1] << "\t\t\t\t"
        << q[2] << "\t\t\t\t" << q[7] << "\t\t\t\t" << q[10] << std::endl;
  }
  if (!out.good()) return fail(CFD_ERR_IO, std::string("write failed: ") + path);
  return CFD_OK;
}

// Initialize(const string &), src/Initialize.cpp:125-176: the state of the physical cells from a
// solution file (rho, p, u, v of each row; U = (rho, rho u, rho v, p/(gamma-1) + rho |V|^2/2) as
// Calculate_Computational_Variables(P, V, Rho, 2) forms it) and the iteration count; ghost rows
// keep the context's current values.  A cell-count mismatch changes nothing (the reference
// reports it and carries on) and returns CFD_ERR_MESH.
cfd_status cfd_read_solution(cfd_ctx *ctx, const char *path, int n_header) {
  if (!ctx || !path || n_header < 0) return fail(CFD_ERR_BAD_ARG, "bad argument");
  std::ifstream in(path);
  if (!in.is_open()) return fail(CFD_ERR_IO, std::string("cannot open ") + path);
  const int NP = ctx->NP, NT = ctx->NT;
  for (int k = 0; k < n_header; k++) {
    int h;
    in >> h;
  }
  int n_cells = -1, iters = 0;
  in >> n_cells >> iters;
  if (!in.good()) return fail(CFD_ERR_IO, std::string("bad solution file header: ") + path);
  if (n_cells != NP) return fail(CFD_ERR_MESH, "solution file has " + std::to_string(n_cells) + " cells, mesh " +
                                                   std::to_string(NP));
  std::vector<double> U(4 * (size_t)NT);
  cfd_status s = cfd_download_U(ctx, U.data());
  if (s != CFD_OK) return s;
  for (int c = 0; c < NP; c++) {
    int idx;
    double dtc, Rho, P, T, v1, v2, M, P0;
    in >> idx >> dtc >> Rho >> P >> T >> v1 >> v2 >> M >> P0;
    if (in.fail()) return fail(CFD_ERR_IO, "bad solution row " + std::to_string(c));
    const double vmag = 0.5 * (v1 * v1 + v2 * v2);
    double *u = U.data() + 4 * (size_t)c;
    u[0] = Rho;
    u[1] = Rho * v1;
    u[2] = Rho * v2;
    u[3] = ((P / kGM1) + Rho * vmag);
  }
  if ((s = cfd_upload_state(ctx, U.data(), NT)) != CFD_OK) return s;
  ctx->launches += launch_set_ctl(ctx->stream, ctx->ds, CTL_ITER, static_cast<double>(iters));
  CUDA_TRY(cudaGetLastError());
  return sync_status(ctx, nullptr);
}

cfd_status cfd_get_min_dt(cfd_ctx *ctx, double *min_dt) {
  if (!ctx || !min_dt) return fail(CFD_ERR_BAD_ARG, "null argument");
  cfd_status s = sync_status(ctx, nullptr);
  *min_dt = ctx->h_ctl[CTL_DTMIN];
  return s;
}

cfd_status cfd_download(cfd_ctx *ctx, double *U, double *prim, double *dt, double *net, double *delu) {
  if (!ctx) return fail(CFD_ERR_BAD_ARG, "null context");
  const int NP = ctx->NP, NT = ctx->NT;
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  std::vector<double> hU(4 * (size_t)NT), hS, hP;
  CUDA_TRY(cudaMemcpy(hU.data(), ctx->ds.U, hU.size() * sizeof(double), cudaMemcpyDeviceToHost));
  if (U) {
    cfd_status su = cfd_download_U(ctx, U);
    if (su != CFD_OK) return su;
  }
  if (prim) {
    hP.resize(5 * (size_t)NT);
    CUDA_TRY(cudaMemcpy(hP.data(), ctx->ds.prim, hP.size() * sizeof(double), cudaMemcpyDeviceToHost));
    if (ctx->prim_from_S) {
      hS.resize(4 * (size_t)NP);
      CUDA_TRY(cudaMemcpy(hS.data(), ctx->ds.S, hS.size() * sizeof(double), cudaMemcpyDeviceToHost));
    }
    for (int i = 0; i < NT; i++) {
      const int r = i < NP ? ctx->perm[i] : i;
      const double rho = hP[i], u = hP[(size_t)NT + i], v = hP[2 * (size_t)NT + i], p = hP[3 * (size_t)NT + i],
                   a = hP[4 * (size_t)NT + i];
      const double E = (ctx->prim_from_S && i < NP) ? hS[3 * (size_t)NP + i] : hU[3 * (size_t)NT + i];
      // The remaining slots of src/Basic_Functions.cpp:162-219 from the stored ones.
      const double inv = 1.0 / rho;
      const double T = (p * inv / 287.0);
      const double vmag = (u * u + v * v);
      const double M = std::sqrt(vmag) / a;
      double *o = prim + 11 * (size_t)r;
      o[0] = rho;
      o[1] = u;
      o[2] = v;
      o[3] = T;
      o[4] = p;
      o[5] = a;
      o[6] = E;
      o[7] = M;
      o[8] = 0.0;
      o[9] = 0.0;
      o[10] = p * std::pow((1.0 + 0.5 * kGM1 * M * M), kGamma1);
    }
  }
  auto fetch_np = [&](const double *src, int ncomp, double *dst) -> cfd_status {
    std::vector<double> h((size_t)ncomp * NP);
    CUDA_TRY(cudaMemcpy(h.data(), src, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (int i = 0; i < NP; i++) {
      const int r = ctx->perm[i];
      for (int k = 0; k < ncomp; k++) dst[(size_t)ncomp * r + k] = h[(size_t)k * NP + i];
    }
    return CFD_OK;
  };
  cfd_status s;
  if (dt && (s = fetch_np(ctx->ds.dtc, 1, dt)) != CFD_OK) return s;
  if (net && (s = fetch_np(ctx->ds.R, 4, net)) != CFD_OK) return s;
  if (delu && (s = fetch_np(ctx->ds.dU, 4, delu)) != CFD_OK) return s;
  return CFD_OK;
}

cfd_status cfd_download_stage_state(cfd_ctx *ctx, double *S) {
  if (!ctx || !S) return fail(CFD_ERR_BAD_ARG, "null argument");
  const int NP = ctx->NP;
  std::vector<double> h(4 * (size_t)NP);
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  CUDA_TRY(cudaMemcpy(h.data(), ctx->ds.S, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
  for (int i = 0; i < NP; i++) {
    const int r = ctx->perm[i];
    for (int k = 0; k < 4; k++) S[4 * (size_t)r + k] = h[(size_t)k * NP + i];
  }
  return CFD_OK;
}

cfd_status cfd_gradient(cfd_ctx *ctx, int var, double *grad) {
  if (!ctx || !grad) return fail(CFD_ERR_BAD_ARG, "null argument");
  const int map[6] = {0, 1, 2, -1, 3, 4};
  if (var < 0 || var > 5 || map[var] < 0) return fail(CFD_ERR_BAD_ARG, "gradient slot must be 0,1,2,4 or 5");
  const int NP = ctx->NP;
  double *dg = nullptr;
  CUDA_TRY(cudaMalloc(&dg, 2 * (size_t)NP * sizeof(double)));
  ctx->launches += launch_gradient(ctx->stream, ctx->dm, ctx->ds, map[var], dg);
  std::vector<double> h(2 * (size_t)NP);
  cudaError_t e = cudaMemcpyAsync(h.data(), dg, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(dg);
  if (e != cudaSuccess) return fail(CFD_ERR_CUDA, cudaGetErrorString(e));
  for (int i = 0; i < NP; i++) {
    const int r = ctx->perm[i];
    grad[2 * (size_t)r] = h[2 * (size_t)i];
    grad[2 * (size_t)r + 1] = h[2 * (size_t)i + 1];
  }
  return CFD_OK;
}

cfd_status cfd_amr_tags(cfd_ctx *ctx, double threshold, double max_fraction, double *indicator, uint8_t *tags) {
  if (!ctx) return fail(CFD_ERR_BAD_ARG, "null context");
  const int NP = ctx->NP;
  if (!ctx->d_amr) {
    // indicator [NP] doubles + tags [NP] bytes + select scratch (2 states + 256 counters)
    const size_t bytes = (size_t)NP * sizeof(double) + (((size_t)NP + 255) & ~size_t(255)) + 2048;
    cfd_status s = ctx_alloc(ctx, &ctx->d_amr, bytes);
    if (s != CFD_OK) return s;
  }
  double *dind = static_cast<double *>(ctx->d_amr);
  uint8_t *dtag = reinterpret_cast<uint8_t *>(dind + NP);
  void *scratch = dtag + (((size_t)NP + 255) & ~size_t(255));
  ctx->launches += launch_amr_indicator(ctx->stream, ctx->dm, ctx->ds, dind);
  if (tags) ctx->launches += launch_amr_tags(ctx->stream, dind, ctx->d_perm, NP, threshold, max_fraction, scratch, dtag);
  CUDA_TRY(cudaGetLastError());
  std::vector<double> h(NP);
  std::vector<uint8_t> ht(tags ? NP : 0);
  CUDA_TRY(cudaMemcpyAsync(h.data(), dind, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  if (tags) CUDA_TRY(cudaMemcpyAsync(ht.data(), dtag, ht.size(), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < NP; i++) {
    if (indicator) indicator[ctx->perm[i]] = h[i];
    if (tags) tags[ctx->perm[i]] = ht[i];
  }
  return CFD_OK;
}

// Autotuner: times each combination of the launch options that never change a result bit
// (face-kernel shape, fused gather + stage, per-cell flux lanes) over `steps` graph-replayed
// pseudo-steps of this context's own mesh and state, keeps the fastest, and restores the state
// (every candidate starts from the same state; the solve is not advanced).
cfd_status cfd_autotune(cfd_ctx *ctx, int steps, char *report, size_t report_len) {
  if (!ctx || steps < 1) return fail(CFD_ERR_BAD_ARG, "bad argument");
  DevState &st = ctx->ds;
  const size_t NT = ctx->NT, NP = ctx->NP;
  struct Part {
    double *p;
    size_t n;
  };
  std::vector<Part> parts = {{st.U, 4 * NT}, {st.S, 4 * NP}, {st.prim, 5 * NT}, {st.R, 4 * NP}, {st.dtc, NP},
                             {st.dtk, NP},    {st.dU, 4 * NP}, {st.ctl, (size_t)CTL_SIZE}};
  if (st.Racc) parts.push_back({st.Racc, 4 * NP});
  if (st.q4) parts.push_back({reinterpret_cast<double *>(st.q4), 4 * NT});
  size_t total = 0;
  for (const Part &q : parts) total += q.n;
  double *snap = nullptr;
  CUDA_TRY(cudaMalloc(&snap, total * sizeof(double)));
  auto copy_all = [&](bool save) {
    size_t off = 0;
    for (const Part &q : parts) {
      if (save) cudaMemcpyAsync(snap + off, q.p, q.n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
      else cudaMemcpyAsync(q.p, snap + off, q.n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream);
      off += q.n;
    }
  };
  struct Cand {
    int faces_shape, fuse, lanes, pdl, patch, minb, tile;
    double ms;
  };
  std::vector<Cand> cands;
  if (ctx->dm.NF > 0) {
    for (int f = 0; f < 5; f++)
      for (int g = 0; g < 2; g++)
        for (int p = 0; p < 2; p++) cands.push_back({f, g, ctx->fp.lanes, p, 0, ctx->fp.flux_minb, 0, 0.0});
    if (ctx->dm.npatch > 0)
      for (int p = 0; p < 2; p++)
        cands.push_back({ctx->fp.faces_shape, 1, ctx->fp.lanes, p, 1, ctx->fp.flux_minb, 0, 0.0});
    if (ctx->tile_ok)
      for (int t = 1; t <= (ctx->tile_tma_ok ? 4 : 1); t++)
        for (int p = 0; p < 2; p++)
          cands.push_back({ctx->fp.faces_shape, 1, ctx->fp.lanes, p, 0, ctx->fp.flux_minb, t, 0.0});
  } else {
    const int dz = ctx->fp.dissipation;
    const bool limited = (dz == 3 || dz == 4 || dz == 5) && ctx->fp.second_order && !ctx->fp.weno;
    for (int mb : {1, 6, 8}) {
      if (mb != 1 && !limited) continue;
      cands.push_back({ctx->fp.faces_shape, ctx->fuse_gather, 1, ctx->dm.pdl, 0, mb, 0, 0.0});
    }
    cands.push_back({ctx->fp.faces_shape, ctx->fuse_gather, 4, ctx->dm.pdl, 0, 1, 0, 0.0});
  }
  const int prof = ctx->profile, graph_on = ctx->use_graph;
  ctx->profile = 0;
  ctx->use_graph = 1;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  copy_all(true);
  cfd_status status = CFD_OK;
  for (Cand &cd : cands) {
    ctx->fp.faces_shape = cd.faces_shape;
    ctx->fuse_gather = cd.fuse;
    ctx->fp.lanes = cd.lanes;
    ctx->dm.pdl = cd.pdl;
    ctx->patch_stage = cd.patch;
    ctx->fp.flux_minb = cd.minb;
    ctx->tile_stage = cd.tile;
    drop_graphs(ctx);
    ctx->launches += launch_set_ctl(ctx->stream, st, CTL_TEND, 0.0);
    ctx->launches += launch_set_ctl(ctx->stream, st, CTL_DONE, 0.0);
    if ((status = enqueue_steps(ctx, 2)) != CFD_OK) break;
    cudaEventRecord(e0, ctx->stream);
    if ((status = enqueue_steps(ctx, steps)) != CFD_OK) break;
    cudaEventRecord(e1, ctx->stream);
    if ((status = sync_status(ctx, nullptr)) != CFD_OK) break;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cd.ms = ms / steps;
    copy_all(false);
  }
  copy_all(false);
  cudaStreamSynchronize(ctx->stream);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(snap);
  ctx->profile = prof;
  ctx->use_graph = graph_on;
  drop_graphs(ctx);
  if (status != CFD_OK) return status;
  const Cand *best = &cands[0];
  for (const Cand &cd : cands)
    if (cd.ms < best->ms) best = &cd;
  ctx->fp.faces_shape = best->faces_shape;
  ctx->fuse_gather = best->fuse;
  ctx->fp.lanes = best->lanes;
  ctx->dm.pdl = best->pdl;
  ctx->patch_stage = best->patch;
  ctx->fp.flux_minb = best->minb;
  ctx->tile_stage = best->tile;
  if (report && report_len > 0) {
    std::string r;
    char line[160];
    for (const Cand &cd : cands) {
      snprintf(line, sizeof(line),
               "faces_shape=%d fuse_gather=%d flux_lanes=%d pdl=%d patch_stage=%d flux_minb=%d tile_stage=%d: %.4f "
               "ms/step%s\n",
               cd.faces_shape, cd.fuse, cd.lanes, cd.pdl, cd.patch, cd.minb, cd.tile, cd.ms, &cd == best ? " (chosen)" : "");
      r += line;
    }
    snprintf(report, report_len, "%s", r.c_str());
  }
  return CFD_OK;
}

namespace {
// Device copies of host arrays for the pointwise entry points; freed on scope exit.
struct DevBufs {
  std::vector<void *> p;
  ~DevBufs() {
    for (void *q : p) cudaFree(q);
  }
  double *put(const double *h, size_t n) {
    void *d = nullptr;
    if (cudaMalloc(&d, n * sizeof(double) + 8) != cudaSuccess) return nullptr;
    p.push_back(d);
    if (h && cudaMemcpy(d, h, n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
    return static_cast<double *>(d);
  }
};

cfd_status set_eval_device(int device) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(CFD_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(CFD_ERR_BAD_ARG, "bad device ordinal");
  CUDA_TRY(cudaSetDevice(device));
  return CFD_OK;
}
}  // namespace

cfd_status cfd_eval_limiter(int limiter, const double *a, const double *b, int n, double *out, int device) {
  if (n < 0 || (n > 0 && (!a || !b || !out))) return fail(CFD_ERR_BAD_ARG, "bad argument");
  if (limiter < CFD_LIM_MINMOD || limiter > CFD_LIM_VANALBADA) return fail(CFD_ERR_BAD_ARG, "bad limiter");
  if (n == 0) return CFD_OK;
  cfd_status st = set_eval_device(device);
  if (st != CFD_OK) return st;
  DevBufs d;
  double *da = d.put(a, n), *db = d.put(b, n), *dout = d.put(nullptr, n);
  if (!da || !db || !dout) return fail(CFD_ERR_CUDA, "device buffers");
  launch_eval_limiter(0, limiter, da, db, n, dout);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpy(out, dout, n * sizeof(double), cudaMemcpyDeviceToHost));
  return CFD_OK;
}

cfd_status cfd_eval_face_flux(int scheme, int precision, const double *UL, const double *UR, const double *normals,
                              const double *lengths, int n, double *F, int device) {
  if (n < 0 || (n > 0 && (!UL || !UR || !normals || !lengths || !F))) return fail(CFD_ERR_BAD_ARG, "bad argument");
  if (scheme != CFD_DISS_ROE && scheme != CFD_DISS_AUSM && scheme != CFD_DISS_HLLC && scheme != CFD_DISS_AUSM_GPU)
    return fail(CFD_ERR_BAD_ARG, "bad face-flux scheme");
  if (precision != CFD_PREC_FP64 && precision != CFD_PREC_FP32_FLUX) return fail(CFD_ERR_BAD_ARG, "bad precision");
  if (n == 0) return CFD_OK;
  cfd_status st = set_eval_device(device);
  if (st != CFD_OK) return st;
  DevBufs d;
  double *dl = d.put(UL, 4 * (size_t)n), *dr = d.put(UR, 4 * (size_t)n), *dn = d.put(normals, 2 * (size_t)n),
         *dlen = d.put(lengths, n), *dF = d.put(nullptr, 4 * (size_t)n);
  if (!dl || !dr || !dn || !dlen || !dF) return fail(CFD_ERR_CUDA, "device buffers");
  launch_eval_face_flux(0, scheme, precision, dl, dr, dn, dlen, n, dF);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpy(F, dF, 4 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost));
  return CFD_OK;
}

cfd_status cfd_kernel_time(cfd_ctx *ctx, const char *kernel, double *total_ms, long long *launches) {
  if (!ctx || !kernel || !total_ms || !launches) return fail(CFD_ERR_BAD_ARG, "null argument");
  std::string k(kernel);
  int kind = k == "flux" ? TK_FLUX : k == "stage" ? TK_STAGE : k == "bc" ? TK_BC : k == "gradients" ? TK_GRAD
           : k == "faces" ? TK_FACES : k == "gather_stage" ? TK_GATHER_STAGE : k == "patch" ? TK_PATCH
           : k == "persistent" ? TK_PERSIST
           : k == "tile" ? TK_TILE : -1;
  if (kind < 0) return fail(CFD_ERR_BAD_ARG, "unknown kernel " + k);
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  for (auto &t : ctx->timed) {
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, t.a, t.b));
    ctx->kind_ms[t.kind] += ms;
    ctx->kind_n[t.kind] += 1;
    cudaEventDestroy(t.a);
    cudaEventDestroy(t.b);
  }
  ctx->timed.clear();
  *total_ms = ctx->kind_ms[kind];
  *launches = ctx->kind_n[kind];
  return CFD_OK;
}

// ------------------------------------ batched solves --------------------------------------
// Many independent meshes run as one union mesh (instance after instance, no renumbering) through
// the same kernels; work lists restrict every launch to the cells, faces, boundary entries and
// record rows of the instances that have not converged yet.
struct cfd_batch {
  int n = 0;
  cfd_ctx *ctx = nullptr;
  std::vector<int> cs, ce, fs, fe, bs, be, gs, ge;  // per-instance ranges in the union
  std::vector<uint8_t> active;
  int *d_start = nullptr, *d_end = nullptr;
  double *d_res = nullptr;
  int table_cap[4] = {0, 0, 0, 0};
  double4 *d_bstate = nullptr;
  double *d_bexit = nullptr;
  std::vector<double> r0_fixed;  // per-instance residual normalisers (empty: first-step residual)
  double diverge = 0.0;          // > 0: an instance whose residual ratio exceeds it stops (steps_to_tol -2)
};

static cfd_status batch_tables(cfd_batch *b) {
  std::vector<int2> t[4];
  auto chunks = [](std::vector<int2> &v, int a, int e, int w) {
    for (int x = a; x < e; x += w) v.push_back(make_int2(x, std::min(x + w, e)));
  };
  for (int i = 0; i < b->n; i++) {
    if (!b->active[i]) continue;
    chunks(t[0], b->cs[i], b->ce[i], kWorkCellBlock);
    chunks(t[1], b->fs[i], b->fe[i], kWorkFaceBlock);
    chunks(t[2], b->bs[i], b->be[i], kWorkItemBlock);
    chunks(t[3], b->cs[i], b->ce[i], kWorkItemBlock);
    chunks(t[3], b->gs[i], b->ge[i], kWorkItemBlock);
  }
  cfd_ctx *ctx = b->ctx;
  int2 *base = ctx->d_tables;
  int2 *p[4];
  size_t off = 0;
  for (int k = 0; k < 4; k++) {
    p[k] = base + off;
    off += b->table_cap[k];
    if (!t[k].empty())
      CUDA_TRY(cudaMemcpyAsync(p[k], t[k].data(), t[k].size() * sizeof(int2), cudaMemcpyHostToDevice, ctx->stream));
  }
  ctx->dm.cblk = p[0];
  ctx->dm.n_cblk = static_cast<int>(t[0].size());
  ctx->dm.fblk = p[1];
  ctx->dm.n_fblk = static_cast<int>(t[1].size());
  ctx->dm.bblk = p[2];
  ctx->dm.n_bblk = static_cast<int>(t[2].size());
  ctx->dm.rblk = p[3];
  ctx->dm.n_rblk = static_cast<int>(t[3].size());
  drop_graphs(ctx);
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return CFD_OK;
}

void cfd_batch_destroy(cfd_batch *b) {
  if (!b) return;
  cfd_destroy(b->ctx);
  delete b;
}

cfd_status cfd_batch_create(int n, const cfd_mesh_desc *meshes, const double *inflow, const cfd_config *cfg,
                            cfd_batch **out) {
  if (n <= 0 || !meshes || !cfg || !out) return fail(CFD_ERR_BAD_ARG, "bad argument");
  if (!(cfg->muscl && cfg->is_second_order)) return fail(CFD_ERR_BAD_ARG, "batched solves use the gradient-MUSCL form");
  if (cfg->reorder) return fail(CFD_ERR_BAD_ARG, "batched solves keep each instance's own numbering (reorder = 0)");
  *out = nullptr;
  long long NPt = 0, NGt = 0, NBt = 0;
  for (int i = 0; i < n; i++) {
    NPt += meshes[i].n_physical;
    NGt += meshes[i].n_ghost;
    NBt += meshes[i].n_boundary;
  }
  if (NPt + NGt > 2000000000LL) return fail(CFD_ERR_BAD_ARG, "batch too large");
  cfd_batch *b = new cfd_batch;
  b->n = n;
  std::vector<int> nf, nbr, bnd;
  std::vector<double> nrm, len, ccd, cvec, area, inva, bstate;
  nf.reserve(NPt);
  int offP = 0, offG = 0, offF = 0;
  for (int i = 0; i < n; i++) {
    const cfd_mesh_desc &d = meshes[i];
    const int NP = d.n_physical;
    if (!d.center_vectors || !d.center_distances) {
      delete b;
      return fail(CFD_ERR_BAD_ARG, "instance " + std::to_string(i) + " lacks centre vectors");
    }
    auto map = [&](int id) { return id < NP ? offP + id : static_cast<int>(NPt) + offG + (id - NP); };
    int nfi = 0;
    for (int c = 0; c < NP; c++) {
      nf.push_back(d.n_faces[c]);
      area.push_back(d.area[c]);
      inva.push_back(d.inv_area[c]);
      for (int f = 0; f < 4; f++) {
        const bool has = f < d.n_faces[c];
        const int N = d.neighbours[4 * c + f];
        nbr.push_back(has ? map(N) : -1);
        if (has && (N >= NP || N > c)) nfi++;
      }
      for (int k = 0; k < 8; k++) {
        nrm.push_back(d.face_normals[8 * c + k]);
        cvec.push_back(d.center_vectors[8 * c + k]);
      }
      for (int k = 0; k < 4; k++) {
        len.push_back(d.face_lengths[4 * c + k]);
        ccd.push_back(d.center_distances[4 * c + k]);
      }
    }
    b->bs.push_back(static_cast<int>(bnd.size() / 4));
    for (int e = 0; e < d.n_boundary; e++) {
      const int *x = d.boundary + 4 * e;
      bnd.insert(bnd.end(), {x[0], offP + x[1], x[2], map(x[3])});
      for (int k = 0; k < 4; k++) bstate.push_back(inflow ? inflow[4 * i + k] : 0.0);
    }
    b->be.push_back(static_cast<int>(bnd.size() / 4));
    b->cs.push_back(offP);
    b->ce.push_back(offP + NP);
    b->gs.push_back(static_cast<int>(NPt) + offG);
    b->ge.push_back(static_cast<int>(NPt) + offG + d.n_ghost);
    b->fs.push_back(offF);
    b->fe.push_back(offF + nfi);
    offP += NP;
    offG += d.n_ghost;
    offF += nfi;
  }
  cfd_mesh_desc u = {static_cast<int>(NPt), static_cast<int>(NGt), nf.data(), nbr.data(), nrm.data(), len.data(),
                     ccd.data(), cvec.data(), area.data(), inva.data(), static_cast<int>(bnd.size() / 4), bnd.data()};
  cfd_status s = cfd_create(&u, cfg, &b->ctx);
  if (s != CFD_OK) {
    delete b;
    return s;
  }
  cfd_ctx *ctx = b->ctx;
  if (ctx->dm.NF != offF) {
    cfd_batch_destroy(b);
    return fail(CFD_ERR_MESH, "face count mismatch in the batch union");
  }
  std::vector<double4> bs4(bnd.size() / 4);
  for (size_t e = 0; e < bs4.size(); e++) bs4[e] = make_double4(bstate[4 * e], bstate[4 * e + 1], bstate[4 * e + 2], bstate[4 * e + 3]);
  if ((s = ctx_upload(ctx, &b->d_bstate, bs4)) != CFD_OK) {
    cfd_batch_destroy(b);
    return s;
  }
  ctx->dm.bstate = inflow ? b->d_bstate : nullptr;
  if ((s = ctx_upload(ctx, &b->d_start, b->cs)) != CFD_OK || (s = ctx_upload(ctx, &b->d_end, b->ce)) != CFD_OK ||
      (s = ctx_alloc(ctx, (void **)&b->d_res, sizeof(double) * n)) != CFD_OK) {
    cfd_batch_destroy(b);
    return s;
  }
  // Work-list capacity: every instance active.
  long long cap[4] = {0, 0, 0, 0};
  for (int i = 0; i < n; i++) {
    cap[0] += (b->ce[i] - b->cs[i] + kWorkCellBlock - 1) / kWorkCellBlock;
    cap[1] += (b->fe[i] - b->fs[i] + kWorkFaceBlock - 1) / kWorkFaceBlock;
    cap[2] += (b->be[i] - b->bs[i] + kWorkItemBlock - 1) / kWorkItemBlock;
    cap[3] += (b->ce[i] - b->cs[i] + kWorkItemBlock - 1) / kWorkItemBlock + (b->ge[i] - b->gs[i] + kWorkItemBlock - 1) / kWorkItemBlock;
  }
  for (int k = 0; k < 4; k++) b->table_cap[k] = static_cast<int>(cap[k]);
  if ((s = ctx_alloc(ctx, (void **)&ctx->d_tables, sizeof(int2) * (cap[0] + cap[1] + cap[2] + cap[3]))) != CFD_OK) {
    cfd_batch_destroy(b);
    return s;
  }
  b->active.assign(n, 1);
  if ((s = batch_tables(b)) != CFD_OK) {
    cfd_batch_destroy(b);
    return s;
  }
  *out = b;
  return CFD_OK;
}

cfd_status cfd_batch_upload_state(cfd_batch *b, const double *U) {
  if (!b || !U) return fail(CFD_ERR_BAD_ARG, "null argument");
  // Instance-ordered rows (each instance: NP_i physical rows then NG_i ghost rows) -> union order.
  const cfd_ctx *ctx = b->ctx;
  std::vector<double> u(4 * (size_t)ctx->NT);
  size_t row = 0;
  for (int i = 0; i < b->n; i++) {
    for (int c = b->cs[i]; c < b->ce[i]; c++, row++)
      for (int k = 0; k < 4; k++) u[4 * (size_t)c + k] = U[4 * row + k];
    for (int g = b->gs[i]; g < b->ge[i]; g++, row++)
      for (int k = 0; k < 4; k++) u[4 * (size_t)g + k] = U[4 * row + k];
  }
  cfd_status s = cfd_upload_state(b->ctx, u.data(), ctx->NT);
  if (s != CFD_OK) return s;
  // A new state restarts every instance.
  b->active.assign(b->n, 1);
  return batch_tables(b);
}

cfd_status cfd_batch_set_boundary_values(cfd_batch *b, const double *inlet, const double *exit_p) {
  if (!b) return fail(CFD_ERR_BAD_ARG, "null argument");
  cfd_ctx *ctx = b->ctx;
  cfd_status s;
  if (inlet) {
    std::vector<double4> v;
    for (int i = 0; i < b->n; i++)
      for (int e = b->bs[i]; e < b->be[i]; e++)
        v.push_back(make_double4(inlet[4 * i], inlet[4 * i + 1], inlet[4 * i + 2], inlet[4 * i + 3]));
    if (!b->d_bstate && (s = ctx_alloc(ctx, (void **)&b->d_bstate, sizeof(double4) * v.size())) != CFD_OK) return s;
    CUDA_TRY(cudaMemcpy(b->d_bstate, v.data(), sizeof(double4) * v.size(), cudaMemcpyHostToDevice));
    ctx->dm.bstate = b->d_bstate;
  }
  if (exit_p) {
    std::vector<double> v;
    for (int i = 0; i < b->n; i++)
      for (int e = b->bs[i]; e < b->be[i]; e++) v.push_back(exit_p[i]);
    if (!b->d_bexit && (s = ctx_alloc(ctx, (void **)&b->d_bexit, sizeof(double) * v.size())) != CFD_OK) return s;
    CUDA_TRY(cudaMemcpy(b->d_bexit, v.data(), sizeof(double) * v.size(), cudaMemcpyHostToDevice));
    ctx->dm.bexit = b->d_bexit;
  }
  drop_graphs(ctx);
  return CFD_OK;
}

cfd_status cfd_batch_set_reference_residual(cfd_batch *b, const double *r0) {
  if (!b) return fail(CFD_ERR_BAD_ARG, "null argument");
  if (r0) b->r0_fixed.assign(r0, r0 + b->n);
  else b->r0_fixed.clear();
  return CFD_OK;
}

cfd_status cfd_batch_download_state(cfd_batch *b, double *U) {
  if (!b || !U) return fail(CFD_ERR_BAD_ARG, "null argument");
  const cfd_ctx *ctx = b->ctx;
  std::vector<double> u(4 * (size_t)ctx->NT);
  cfd_status s = cfd_download_U(b->ctx, u.data());
  if (s != CFD_OK) return s;
  size_t row = 0;
  for (int i = 0; i < b->n; i++) {
    for (int c = b->cs[i]; c < b->ce[i]; c++, row++)
      for (int k = 0; k < 4; k++) U[4 * row + k] = u[4 * (size_t)c + k];
    for (int g = b->gs[i]; g < b->ge[i]; g++, row++)
      for (int k = 0; k < 4; k++) U[4 * row + k] = u[4 * (size_t)g + k];
  }
  return CFD_OK;
}

static cfd_status batch_residuals(cfd_batch *b, std::vector<double> &res) {
  cfd_ctx *ctx = b->ctx;
  ctx->launches += launch_instance_residual(ctx->stream, ctx->ds, ctx->NP, b->d_start, b->d_end, b->n, b->d_res);
  res.resize(b->n);
  CUDA_TRY(cudaMemcpyAsync(res.data(), b->d_res, sizeof(double) * b->n, cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  for (double &r : res) r = std::sqrt(r);
  return CFD_OK;
}

cfd_status cfd_batch_residuals(cfd_batch *b, double *res) {
  if (!b || !res) return fail(CFD_ERR_BAD_ARG, "null argument");
  std::vector<double> r;
  cfd_status s = batch_residuals(b, r);
  if (s != CFD_OK) return s;
  for (int i = 0; i < b->n; i++) res[i] = r[i];
  return CFD_OK;
}

cfd_status cfd_batch_set_option(cfd_batch *b, const char *name, double value) {
  if (!b || !name) return fail(CFD_ERR_BAD_ARG, "null argument");
  if (std::string(name) == "divergence_ratio") {
    if (!(value >= 0.0)) return fail(CFD_ERR_BAD_ARG, "divergence_ratio must be >= 0");
    b->diverge = value;
    return CFD_OK;
  }
  return cfd_set_option(b->ctx, name, value);
}

cfd_status cfd_batch_run(cfd_batch *b, int max_steps, double tol, int check_every, int *steps_to_tol,
                         double *time_to_tol, double *res_ratio, long long *cell_updates, int *steps_done) {
  if (!b || max_steps < 1 || check_every < 1) return fail(CFD_ERR_BAD_ARG, "bad argument");
  cfd_ctx *ctx = b->ctx;
  const int n = b->n;
  std::vector<double> r0, r;
  std::vector<int> sto(n, -1);
  std::vector<double> tto(n, -1.0), ratio(n, 1.0);
  auto now = [] {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
  };
  cfd_status s;
  long long cu = 0;
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  const double t0 = now();
  if ((s = enqueue_steps(ctx, 1)) != CFD_OK) return s;
  for (int i = 0; i < n; i++)
    if (b->active[i]) cu += b->ce[i] - b->cs[i];
  if ((s = batch_residuals(b, r0)) != CFD_OK) return s;
  if (!b->r0_fixed.empty()) r0 = b->r0_fixed;
  int steps = 1;
  while (steps < max_steps) {
    bool any = false;
    for (int i = 0; i < n; i++) any = any || b->active[i];
    if (!any) break;
    const int k = std::min(check_every, max_steps - steps);
    if ((s = enqueue_steps(ctx, k)) != CFD_OK) return s;
    steps += k;
    long long act = 0;
    for (int i = 0; i < n; i++)
      if (b->active[i]) act += b->ce[i] - b->cs[i];
    cu += act * k;
    if ((s = batch_residuals(b, r)) != CFD_OK) return s;
    const double t = now() - t0;
    bool changed = false;
    for (int i = 0; i < n; i++) {
      if (!b->active[i]) continue;
      ratio[i] = r0[i] > 0.0 ? r[i] / r0[i] : 0.0;
      if (!(ratio[i] > tol)) {
        b->active[i] = 0;
        sto[i] = steps;
        tto[i] = t;
        changed = true;
      } else if (b->diverge > 0.0 && ratio[i] > b->diverge) {
        b->active[i] = 0;  // residual growth: the instance stops, the caller falls back
        sto[i] = -2;
        changed = true;
      }
    }
    if (changed && (s = batch_tables(b)) != CFD_OK) return s;
  }
  if ((s = sync_status(ctx, nullptr)) != CFD_OK) return s;
  for (int i = 0; i < n; i++) {
    if (steps_to_tol) steps_to_tol[i] = sto[i];
    if (time_to_tol) time_to_tol[i] = tto[i];
    if (res_ratio) res_ratio[i] = ratio[i];
  }
  if (cell_updates) *cell_updates = cu;
  if (steps_done) *steps_done = steps;
  return CFD_OK;
}

long long cfd_kernel_launches(const cfd_ctx *ctx) { return ctx ? ctx->launches : 0; }
int cfd_face_count(const cfd_ctx *ctx) { return ctx ? ctx->dm.NF : 0; }
size_t cfd_device_bytes(const cfd_ctx *ctx) { return ctx ? ctx->bytes : 0; }

}  // extern "C"
