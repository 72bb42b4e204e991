// Device data layout and kernel declarations of the residual/update path.
//
// HBM layout (all arrays in device cell order; physical cells 0..NP-1 possibly renumbered (RCM or
// patches), ghost cells NP..NT-1 in the reference's ghost order):
//   geometry, face-major SoA [4][NP]: nbr, nx, ny, dl; limiter stencil n2, d1l, d2l; centre vectors;
//   the neighbour and face-table slots again as one int4 per cell (nbr4, cface4); per unique face
//   also its owner and neighbour as one int2 (fon) and nx, ny, dl, dx as one double4 (fg4)
//   per cell [NP]: nf, area, inv_area, degenerate-face mask; boundary entries per cell (CSR)
//   unique faces [NF] (face-based forms): owner, neighbour, owner-side geometry; cell slot -> face
//   state, component-major SoA: U[4][NT] (U^n on physical rows, boundary values on ghost rows),
//   S[4][NP] (RK stage state), prim[5][NT] (rho, u, v, p, a), R[4][NP] (net flux),
//   dtc[NP] (Cell::del_t), dU[4][NP] (Cells_DelU); face-based forms: the primitives again as
//   q4[NT] (rho, u, v, p), gradients rec[NP][8] and face fluxes F[NF]
#pragma once
#include <vector>
#include <cuda.h>  // CUtensorMap (the tensor maps of the TMA tile form; no driver library is linked)
#include <cuda_runtime.h>
#include <stdint.h>

namespace cfdb {

// One face of a patch (64 B, so one record is one aligned load set): the neighbour cell, the
// shared-memory rows of its two cells (owner | neighbour << 16; 0xFFFF = ghost neighbour), the
// face slots it fills (owner | neighbour << 8; 0xFF = not a cell of the patch), and the face's
// owner-side normal, length and centre-to-centre vector.
struct PatchFace {
  int N, rows, slots, face;
  double nx, ny, dl, dx, dy, pad;
};

struct DevMesh {
  int NP, NT, NB;
  const int *nf;
  const int *nbr;
  const double *nx, *ny, *dl;
  const double *area, *inv_area;
  const int *n2;
  const double *d1l, *d2l;
  const double *cvx, *cvy;  // [4][NP] centre-to-centre vectors (gradient MUSCL)
  const uint8_t *degen;
  const int4 *bnd;  // kind, cell, face, ghost
  const int *bptr, *bidx;  // boundary entries of each cell: bidx[bptr[c] .. bptr[c + 1]) (CSR)
  // Unique faces (face-based forms): owner and neighbour cell, owner-side geometry, and for each
  // cell slot the face id (owner side) or -(id + 1) (neighbour side).
  int NF;
  const int *fo, *fn;
  const double *fnx, *fny, *fdl, *fdx, *fdy;
  const int *cface;  // [4][NP]
  const int2 *fon;     // [NF] owner, neighbour of each face (one load)
  const double4 *fg4;  // [NF] nx, ny, dl, dx of each face (dy stays in fdy)
  const int4 *cface4;  // [NP] the same four slots per cell (one 16-byte load)
  const int4 *nbr4;    // [NP] the four neighbour slots per cell
  // Optional work lists (batched solves): each entry is one thread block's [start, end) range of
  // cells (128 per block), faces (128), boundary entries (256) or record rows (256, physical and
  // ghost rows); null = all items.
  const int2 *cblk, *fblk, *bblk, *rblk;
  int n_cblk, n_fblk, n_bblk, n_rblk;
  // Launch policy: 1 = the kernels of a pseudo-step are launched with programmatic stream
  // serialization (each waits on its predecessor grid before touching memory).
  int pdl;
  // Per boundary entry (batched solves), or null: inlet values read by the inlet kind
  // (CFD_INLET_FIXED and CFD_INLET_FARFIELD: rho, u, v, p; CFD_INLET_TOTAL_PT: p0, T0) and the
  // exit pressure (CFD_EXIT_STATIC_P, CFD_EXIT_FIXED_P_REF).
  const double4 *bstate;
  const double *bexit;
  // Patch form (face-based, per-cell dt; single solves): thread block b owns the cells
  // [patch[b].x, patch[b].x + patch[b].y) (at most kPatchCells, contiguous in device order),
  // recomputes the records of its halo cells phcell[phptr[b] .. phptr[b + 1]) and evaluates the
  // faces pface[pfptr[b] .. pfptr[b + 1]) that touch its cells (rows: own cells first, then
  // halo).  patch_rows = the largest own + halo row count (row stride of the shared records).
  int npatch, patch_rows;
  const int2 *patch;
  // Blocks of k_gather_stage resident on the whole device at once (SMs x blocks per SM): the grid
  // of its reducing stage (0 = one block per 128 cells).
  int wave_blocks;
  // L2 access-policy window given to every launch (null / 0: none): the (rho, u, v, p) rows and the
  // face-flux array that follows them, kept as persisting lines between the kernels of a stage.
  void *l2_base;
  size_t l2_bytes;
  float l2_hit;
  const int *phptr, *phcell, *pfptr;
  const PatchFace *pface;
};

constexpr int kPatchCells = 128;

constexpr int kWorkCellBlock = 128;
constexpr int kMaxGroups = 256;  // block groups of the two-level grid reductions
constexpr int kWorkItemBlock = 256;
constexpr int kWorkFaceBlock = 128;  // faces per work-list entry (the face kernel's 128-thread shapes)

struct DevState {
  double *U;     // [4][NT]
  double *S;     // [4][NP]
  double *prim;  // [5][NT]
  double *R;     // [4][NP]
  double *Racc;  // [4][NP] (RK4 accumulator)
  double *dtc;   // [NP]
  double *dtk;   // [NP] dt kept for the whole step (RK4 / SSP with LTS)
  double *dU;    // [4][NP]
  double *rec;   // [NP][8] Green-Gauss gradients (x, y) of rho, u, v, p (face-based forms),
                 // 64 B = 2 x 32 B per cell
  double4 *q4;   // [NT] (rho, u, v, p) of every row, written wherever the primitives are, so the
                 // face-based kernels fetch a neighbour's state with one 32-byte load (or null)
  float4 *recf;  // [NP][2] the gradients rounded to float, in place of rec, for the FP32-flux form
                 // (whose face kernel rounds them to float anyway), or null
  double4 *F;    // [NF] face fluxes (face-based forms)
  // reduction / control block (see CtrlIdx)
  double *ctl;
  double *partial;     // [(nblk_max + kMaxGroups) * 9]
  unsigned int *counter;
  unsigned int *gcount;  // [kMaxGroups + 1] group and top counters of two-level reductions
  int *status;         // [0] status code, [1] first bad cell (device order)
};

// Slots of the device control block `ctl`.
enum CtrlIdx : int {
  CTL_DTMIN = 0,       // Min_dt of the last flux evaluation
  CTL_DTSTEP = 1,      // dt frozen for the current step (RK4 / SSP-RK3)
  CTL_TOTAL_TIME = 2,  // Total_Time
  CTL_ITER = 3,        // iterations (as double)
  CTL_DONE = 4,        // 1 when Total_Time >= t_end
  CTL_TEND = 5,        // t_end (<= 0: none)
  CTL_ERR = 8,         // Error[0..3]
  CTL_RES = 12,        // plain ||R||_2 [4]
  CTL_SIZE = 16
};

struct FluxParams {
  int dissipation;      // 1 LLF, 2 MOVERS, 3 ROE, 4 RICCA, 5 MOVERS_NWSC, 6 AUSM, 7 HLLC
  int movers_single;    // MOVERS: the energy component's alpha for all four (the reference's Is_MOVERS_1)
  int movers_efix;      // MOVERS: entropy fix of alpha (the reference's Enable_Entropy_Fix)
  int second_order;
  int limiter;
  int recon_prim;
  int muscl;            // 0 reference stencil, 1 Green-Gauss-gradient MUSCL
  int lanes;            // threads per cell in the flux kernel: 1 or 4
  int flux_minb = 1;    // one-lane limited second-order kernels built for 1, 6 or 8 resident blocks per SM
  int persist_minb = 0;  // persistent stage kernel built for 4, 6 or 8 resident blocks per SM (0: 6 in
                         // FP64, 8 in the FP32-flux form)
  int faces_shape;      // face kernel launch: 0 256 threads, 1 256 threads at <= 80 registers, 2 128 threads
  int weno;             // 1: the reference's WENO path (Evaluate_Cell_Net_Flux_WENO), quad cells
  int weno_char;        // WENO on characteristic variables (the reference's Is_Char)
  int consistent;       // 1: limiter/LLF/exit read the stage state instead of U^n
  int precision;
  double cfl, zeta, zeta1;
  double eflin;         // entropy fix of the linear waves in the gradient-MUSCL Roe flux (0: off)
  double shock_fix;     // Rusanov dissipation on faces with |grad p| |d| > shock_fix * p (0: off)
};

struct BcParams {
  int inlet_bc, exit_bc;
  double inlet_rho, inlet_p, inlet_u, inlet_v, inlet_p0, inlet_t0, exit_p, r_gas;
};

// Structured-block tables of the tile form (a single block of ni x nj quads numbered
// c = j * ni + i in device order).  The unique faces come in two structured families:
// W(i, j) between cells (i - 1, j) and (i, j), i = 0..ni, and S(i, j) between (i, j - 1) and
// (i, j), j = 0..nj; each keeps the values of its unique face (owner-side normal, length and
// centre-to-centre vector) and a flag, 1 when its owner is the cell on the high side (i, j).
// Around each cell the positions p = 0..3 run E, N, W, S (E, S, W, N when lh = 1); the cell's
// face slot f is position (f + r) & 3.  Per cell one byte: r in bits 0-1, and bit 2 + p set
// when the cell owns the face at position p.
constexpr int kTileCellsX = 32, kTileCellsY = 8;  // cells of one tile (one thread block)
struct TileMesh {
  int ni, nj, tiles_i, tiles_j, lh;
  const int *gW, *gE, *gS, *gN;  // ghost rows beside the block's boundary cells: [nj], [nj], [ni], [ni]
  const unsigned char *code;     // [NP]
  const double4 *fw;             // [nj][ni + 1] nx, ny, dl, dx of the W faces
  const double *fwdy;            // [nj][ni + 1] dy
  const unsigned char *fwo;      // [nj][ni + 1] owner on the high side
  const double4 *fs;             // [nj + 1][ni] the same for the S faces
  const double *fsdy;
  const unsigned char *fso;
  // The same face values as 48-byte records (nx, ny, dl, dx, dy, 1.0 when the owner is on the high
  // side else 0.0), [nj][ni + 1] and [nj + 1][ni]: the tensors the TMA tile form loads.
  const double *gw6, *gs6;
  // TMA form: 1 = each block prefetches into L2 the inputs of the tile one wave ahead (option
  // "tile_prefetch", off by default: on B200 the prefetches slowed the face phase more than they
  // shortened the loads).
  int prefetch_ahead;
};

// Tensor maps of the TMA tile form: the (rho, u, v, p) rows of the block as a 3-D tensor
// (4 doubles, ni, nj) with a box of the tile and two rings, and the two face-record tensors
// (6 doubles, ni + 1, nj) and (6 doubles, ni, nj + 1) with boxes of the faces the tile and its
// one-ring halo touch.  Passed by value as a __grid_constant__ kernel parameter.
struct TileMaps {
  CUtensorMap q, gw, gs;
};

// Kernel launchers (stream-ordered, no host synchronisation).  Each returns the number of
// kernels launched.
int launch_prim_all(cudaStream_t s, const DevMesh &m, DevState &st);
int launch_bc(cudaStream_t s, const DevMesh &m, DevState &st, const BcParams &bp, int stage_src_is_S, int cur_is_S);
int launch_flux(cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp, int stage_src_is_S);
// Lax_Fedrichs over cells grouped by wavefront level (cells[level_start[l] .. level_start[l+1])).
int launch_lax_friedrichs(cudaStream_t s, const DevMesh &m, DevState &st, const int *cells,
                          const std::vector<int> &level_start);
// kind: 1,2,3 = reference RK3 stages; 0 = Explicit; 11..14 = RK4 stages; fuse_final = apply
// Estimate_Error + Update in the last stage's kernel.
int launch_stage(cudaStream_t s, const DevMesh &m, DevState &st, int kind, int lts, int fuse_final, int keep_delu);
// Face-based forms with a per-cell stage dt (lts 1 or 2): gradients, face fluxes and the fused
// gather + stage update.
int launch_faces(cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp);
// Persistent form of one face-based stage (batched solves): gradients, faces and gather + update
// in one cooperative launch of `grid` blocks over the work lists, bounded grid barriers between
// the phases (CFD_ERR_TIMEOUT in the status word when a wait runs out).  persistent_grid: the
// largest co-resident grid (0 when cooperative launches are not available).
int persistent_grid(const FluxParams &fp);
int launch_persistent_stage(cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp,
                            const BcParams &bp, int kind, int lts, int fuse_final, int keep_delu, int flags,
                            int with_dt, int with_bc, int grid, unsigned int test_arrivals);
int launch_gather(cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp);
// Fused gather + stage update of the per-cell-dt forms; del_t comes from the gradient pass
// (launch_muscl_gradients with with_dt).  flags: bit 1 the owner thread writes its ghosts for the
// next stage (non-final stages), bit 2 that next stage's supersonic-exit copy reads the stage state.
int launch_gather_stage(cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp, const BcParams &bp,
                        int kind, int lts, int fuse_final, int keep_delu, int flags);
// Patch form of one stage (gradients, face fluxes, gather and stage update in one kernel): reads
// the primitives `prim_in` and writes the stage's primitives and ghosts to st.prim, which must be a
// different buffer (blocks read their halo cells' primitives while others write theirs).  Same
// flags as launch_gather_stage; ghost rows are carried to st.prim at every stage.
int launch_patch_stage(cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp, const BcParams &bp,
                       int kind, int lts, int fuse_final, int keep_delu, int flags, const double *prim_in);
// Tile form of one stage on a structured block (per-cell dt, three-stage integrators): one thread
// block per tile of 32 x 8 cells reads the (rho, u, v, p) rows `q_in` of its cells and two rings
// around them into shared memory, forms the gradients of its cells and of the halo cells beside
// its sides, the fluxes of every face of its cells and the gather + stage update, and writes the
// stage's rows (and the next stage's ghost rows) to st.q4, which must be a different buffer.
// Same flags as launch_gather_stage; with_dt as launch_muscl_gradients.
int launch_tile_stage(cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp, const BcParams &bp,
                      const TileMesh &tm, const double4 *q_in, int kind, int lts, int fuse_final, int keep_delu,
                      int flags, int with_dt);
// Opt-in to the tile kernels' dynamic shared memory (0 if the device cannot give it).
int tile_prepare();
// TMA form of the tile stage (same arguments and results as launch_tile_stage, bit for bit): the
// state rows of the tile and its two rings and the face records of the tile and its halo arrive
// by three cp.async.bulk.tensor loads on one mbarrier, the stage inputs of the tile's cells by
// cp.async, all issued at block start, so the gradient, face and update phases read only shared
// memory.  maps.q must describe q_in.  variant 0: the stage inputs too are prefetched into
// shared memory (256 threads, 2 blocks per SM); 1: they are loaded where used (3 blocks per SM);
// 2: as 0 with 288 threads (two rounds of face fluxes instead of three).  tile_tma_prepare: the
// shared-memory opt-in (0: not available).  tile_tma_boxes: the box extents the host encodes the
// maps with.
int launch_tile_tma(cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp, const BcParams &bp,
                    const TileMesh &tm, const TileMaps &maps, const double4 *q_in, int kind, int lts, int fuse_final,
                    int keep_delu, int flags, int with_dt, int variant);
int tile_tma_prepare();
void tile_tma_boxes(int q[3], int gw[3], int gs[3]);
// Dynamic shared memory of the patch kernel for m.patch_rows, and the opt-in to it (0 if the
// device cannot give it).
size_t patch_smem_bytes(const DevMesh &m);
int patch_prepare(const DevMesh &m);
// SMs x resident blocks of k_gather_stage on the current device (0 if unknown).
int gather_stage_wave_blocks();
int launch_error(cudaStream_t s, const DevMesh &m, DevState &st);
int launch_update(cudaStream_t s, const DevMesh &m, DevState &st, int from_S);
int launch_eval_limiter(cudaStream_t s, int limiter, const double *a, const double *b, int n, double *out);
int launch_eval_face_flux(cudaStream_t s, int scheme, int precision, const double *UL, const double *UR,
                          const double *nrm, const double *len, int n, double *F);
int launch_gradient(cudaStream_t s, const DevMesh &m, DevState &st, int var, double *grad);
// with_dt: also del_t of every physical cell (the fused per-cell-dt forms).  bc (or null): apply
// the boundary conditions of each cell's boundary entries first (the first stage of a step, in
// place of launch_bc; needs every ghost to neighbour only its owner cell).
int launch_muscl_gradients(cudaStream_t s, const DevMesh &m, DevState &st, const FluxParams &fp, int with_dt,
                           const BcParams *bc = nullptr);
int launch_amr_indicator(cudaStream_t s, const DevMesh &m, DevState &st, double *ind);
int launch_set_ctl(cudaStream_t s, DevState &st, int idx, double v);
// TagRefinableCells on the device; scratch holds >= 2 x 32 + 1024 bytes.
int launch_amr_tags(cudaStream_t s, const double *ind, const int *ref, int NP, double threshold, double max_fraction,
                    void *scratch, uint8_t *tags);
int launch_import_aos(cudaStream_t s, const double *aos, const int *perm, int NP, int NT, double *U);
int launch_export_aos(cudaStream_t s, const double *U, const int *perm, int NP, int NT, int ld, double *aos);

int flux_block_count(int NP);
// Per-instance plain residual sum(R_rho^2) over [start[i], end[i]) cell ranges, one block each.
int launch_instance_residual(cudaStream_t s, const DevState &st, int NP, const int *start, const int *end, int n,
                             double *out);

}  // namespace cfdb
