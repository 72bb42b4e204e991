// Test infrastructure only: a C-linkage driver over the UNMODIFIED reference CPU path.
//
// Compiled together with the reference's own src/*.cpp (see oracle/Makefile) into
// oracle/_ref/libcfdref.so.  The tests load it with ctypes and use it as the checker for the
// CUDA path and for the C restatement in oracle/cfd_oracle.c.  Nothing in the product links it.
//
// It reproduces the reference set-up and loop exactly as the reference's driver does it:
//   mesh      Read_VTK_Grid                          src/Read_Gmsh_File.cpp:11-144
//   ghosts    Construct_Ghost_Cells                  src/Grid_Computations.cpp:394-442
//   distances Calculate_Cell_Center_Distances        src/Grid_Computations.cpp:802-827
//   storage   Initialize(const int&)                 src/Initialize.cpp:58-123
//   loop      BC -> RK3 | Explicit -> Estimate_Error -> Update
//                                                    src/Solver.cpp:94-125
// with the harness-only fixes the reference needs to run at all:
//   * ghost Cell::del_t = 1e300 (get_Min_dt scans ghosts whose del_t is never written,
//     src/Numerical_Method.cpp:322-330, include/Globals.h:319,325);
//   * meshes are read through the VTK path only (the .txt reader mis-pairs faces and
//     neighbours, src/Grid_Computations.cpp:150-151 vs :691-727);
//   * explicit boundary triple lists may replace the bounding-box classification
//     (src/Read_Gmsh_File.cpp:490-625) for non-box domains;
//   * the harness stops at a terminating time itself (src/Solver.cpp:127-142 never breaks);
//   * stdout is silenced while the reference prints per-cell / per-face diagnostics.
#include "definitions.h"
#include "Globals.h"
#include "Grid.h"
#include "Flux.h"
#include "Solver.h"
#include "Timestep.h"
#include "Error_Update.h"
#include "Boundary_Conditions.h"
#include "Initialize.h"
#include "Primitive_Computational.h"
#include "Gradients.h"
#include "Weno.h"
#include "IO_Write.h"
#include "Viscous_Functions.h"

#include <algorithm>
#include <cmath>

#include <unistd.h>
#include <fcntl.h>
#include <cstring>

extern V_D Cells_DelT;                  // src/Initialize.cpp:48
extern vector<V_D> Cells_Viscous_Flux;  // src/Initialize.cpp
void Ausm_Flux(const int &Cell_No);     // src/Ausm_Flux.cpp:5 (no header declaration)

// Present only when the B200 drop-in shim is linked in (oracle/_ref/libcfdref_dropin.so).
extern "C" void b200_shim_reset() __attribute__((weak));
extern "C" void b200_shim_sync() __attribute__((weak));
extern "C" void b200_shim_set_sync_every(int) __attribute__((weak));

namespace {
int g_saved_stdout = -1;
// The reference prints per-call diagnostics on stdout; they are discarded unless REFH_VERBOSE is
// set in the environment.
void quiet_begin() {
  if (getenv("REFH_VERBOSE")) return;
  fflush(stdout);
  std::cout.flush();
  g_saved_stdout = dup(1);
  int devnull = open("/dev/null", O_WRONLY);
  dup2(devnull, 1);
  close(devnull);
}
void quiet_end() {
  fflush(stdout);
  std::cout.flush();
  if (g_saved_stdout >= 0) {
    dup2(g_saved_stdout, 1);
    close(g_saved_stdout);
    g_saved_stdout = -1;
  }
}
bool g_finalized = false;
}  // namespace

extern "C" {

// Clears every container the reference grows with push_back so a fresh mesh can be loaded.
void refh_reset() {
  if (b200_shim_reset) b200_shim_reset();
  Cells.clear();
  Boundary_Cells.clear();
  Inlet_Cells_List.clear();
  Exit_Cells_List.clear();
  Wall_Cells_List.clear();
  Symmetry_Cells_List.clear();
  CF.clear();
  Cells_DelT.clear();
  Cells_Net_Flux.clear();
  Cells_DelU.clear();
  Cells_Face_Boundary_Type.clear();
  U_Cells.clear();
  U_Cells_RK_1.clear();
  U_Cells_RK_2.clear();
  Primitive_Cells.clear();
  Cells_Viscous_Flux.clear();
  Gradient_Refinement_Indicator.clear();
  No_Physical_Cells = 0;
  No_Ghost_Cells = 0;
  Total_No_Cells = 0;
  iterations = 0;
  Total_Time = 0.0;
  Min_dt = 0.0;
  g_finalized = false;
  // Solver defaults of the reference globals (zero-initialised statics in the reference).
  NUM_FLUX_COMPONENTS = 4;
  Is_Viscous_Wall = false;
  Is_WENO = false;
  Is_Char = false;
  Is_Implicit_Method = false;
  Non_Dimensional_Form = false;
  Is_Inlet_SubSonic = false;
  Is_Exit_SubSonic = false;
  has_Symmetry_BC = false;
  Enable_AMR = false;
  Test_Case = 1;
}

// Reads a legacy-VTK mesh with the reference reader.  Returns the number of physical cells.
int refh_load_vtk(const char *path) {
  refh_reset();
  quiet_begin();
  bool ok = Read_VTK_Grid(string(path));
  quiet_end();
  return ok ? No_Physical_Cells : -1;
}

// Replaces the bounding-box boundary lists with explicit (cell, face, ghost) triples.
// kind: 0 inlet, 1 exit, 2 wall, 3 symmetry.
void refh_clear_boundary_lists() {
  Inlet_Cells_List.clear();
  Exit_Cells_List.clear();
  Wall_Cells_List.clear();
  Symmetry_Cells_List.clear();
}
void refh_add_boundary(int kind, int cell, int face, int ghost) {
  V_I *l = kind == 0 ? &Inlet_Cells_List : kind == 1 ? &Exit_Cells_List : kind == 2 ? &Wall_Cells_List : &Symmetry_Cells_List;
  l->push_back(cell);
  l->push_back(face);
  l->push_back(ghost);
  if (kind == 3) has_Symmetry_BC = true;
}

// Ghost geometry, centre distances, storage; then the del_t fix for ghosts.
int refh_finalize_mesh() {
  quiet_begin();
  Construct_Ghost_Cells();
  Calculate_Cell_Center_Distances();
  Initialize(Test_Case);
  quiet_end();
  for (int g = No_Physical_Cells; g < Total_No_Cells; g++) Cells[g].del_t = 1e300;
  g_finalized = true;
  return Total_No_Cells;
}

void refh_counts(int *out) {
  out[0] = No_Physical_Cells;
  out[1] = No_Ghost_Cells;
  out[2] = (int)Inlet_Cells_List.size() / 3;
  out[3] = (int)Exit_Cells_List.size() / 3;
  out[4] = (int)Wall_Cells_List.size() / 3;
  out[5] = (int)Symmetry_Cells_List.size() / 3;
}

void refh_get_boundary_list(int kind, int *out) {
  V_I *l = kind == 0 ? &Inlet_Cells_List : kind == 1 ? &Exit_Cells_List : kind == 2 ? &Wall_Cells_List : &Symmetry_Cells_List;
  for (size_t i = 0; i < l->size(); i++) out[i] = (*l)[i];
}

// Geometry in reference order; 4 face slots per cell, unused slots = -1 / 0.
void refh_get_geometry(int *nfaces, int *nbr, double *normals, double *lengths, double *ccd,
                       double *area, double *inv_area, double *centers) {
  for (int c = 0; c < No_Physical_Cells; c++) {
    const Cell &C = Cells[c];
    nfaces[c] = C.numFaces;
    for (int f = 0; f < 4; f++) {
      bool has = f < C.numFaces;
      nbr[4 * c + f] = has ? C.Neighbours[f] : -1;
      normals[8 * c + 2 * f] = has ? C.Face_Normals[2 * f] : 0.0;
      normals[8 * c + 2 * f + 1] = has ? C.Face_Normals[2 * f + 1] : 0.0;
      lengths[4 * c + f] = has ? C.Face_Areas[f] : 0.0;
      ccd[4 * c + f] = has ? C.Cell_Center_Distances[f] : 0.0;
    }
    area[c] = C.Area;
    inv_area[c] = C.Inv_Area;
  }
  for (int c = 0; c < Total_No_Cells; c++) {
    const Cell &C = Cells[c];
    for (int k = 0; k < 3; k++) centers[3 * c + k] = C.Cell_Center.size() == 3 ? C.Cell_Center[k] : 0.0;
  }
}

// Named scalar parameters (the keys of Solver_Config plus the BC flags the JSON never sets).
int refh_set_param(const char *name, double v) {
  string n(name);
  if (n == "Is_Second_Order") Is_Second_Order = v != 0.0;
  else if (n == "Time_Accurate") Time_Accurate = v != 0.0;
  else if (n == "Local_Time_Stepping") Local_Time_Stepping = v != 0.0;
  else if (n == "Dissipation_Type") Dissipation_Type = (int)v;
  else if (n == "Is_MOVERS_1") Is_MOVERS_1 = v != 0.0;
  else if (n == "Enable_Entropy_Fix") Enable_Entropy_Fix = v != 0.0;
  else if (n == "CFL") CFL = v;
  else if (n == "Limiter_Zeta") Limiter_Zeta = v;
  else if (n == "Limiter_Zeta1") Limiter_Zeta1 = v;
  else if (n == "Is_Inlet_SubSonic") Is_Inlet_SubSonic = v != 0.0;
  else if (n == "Is_Exit_SubSonic") Is_Exit_SubSonic = v != 0.0;
  else if (n == "has_Symmetry_BC") has_Symmetry_BC = v != 0.0;
  else if (n == "Inlet_Rho") inletCond.Rho = v;
  else if (n == "Inlet_P") inletCond.P = v;
  else if (n == "Inlet_u") inletCond.u = v;
  else if (n == "Inlet_v") inletCond.v = v;
  else if (n == "Is_WENO") Is_WENO = v != 0.0;
  else if (n == "Is_Char") Is_Char = v != 0.0;
  else if (n == "Enable_AMR") Enable_AMR = v != 0.0;
  else if (n == "AMR_Period") AMR_Period = (int)v;
  else if (n == "AMR_Gradient_Threshold") AMR_Gradient_Threshold = v;
  else if (n == "AMR_Max_Fraction") AMR_Max_Fraction = v;
  else return -1;
  return 0;
}

// Sets U for cells [0, n) and their primitives through the reference EOS
// (src/Basic_Functions.cpp:100-156), as Initialize_TestCase does (src/Initialize_TestCase.cpp:47-57).
void refh_set_state(const double *U, int n) {
  for (int c = 0; c < n; c++) {
    for (int k = 0; k < 4; k++) U_Cells[c][k] = U[4 * c + k];
    Calculate_Primitive_Variables(c, U_Cells[c]);
    for (int k = 0; k < 11; k++) Primitive_Cells[c][k] = Global_Primitive[k];
  }
}

// Overwrites one primitive slot directly (used to plant states between stages in unit tests).
void refh_set_primitive(const double *P, int n) {
  for (int c = 0; c < n; c++)
    for (int k = 0; k < 11; k++) Primitive_Cells[c][k] = P[11 * c + k];
}

void refh_get_U(double *out) {
  for (int c = 0; c < Total_No_Cells; c++)
    for (int k = 0; k < 4; k++) out[4 * c + k] = U_Cells[c][k];
}
void refh_get_prim(double *out) {
  for (int c = 0; c < Total_No_Cells; c++)
    for (int k = 0; k < 11; k++) out[11 * c + k] = Primitive_Cells[c][k];
}
void refh_get_net_flux(double *out) {
  for (int c = 0; c < No_Physical_Cells; c++)
    for (int k = 0; k < 4; k++) out[4 * c + k] = Cells_Net_Flux[c][k];
}
void refh_get_delU(double *out) {
  for (int c = 0; c < No_Physical_Cells; c++)
    for (int k = 0; k < 4; k++) out[4 * c + k] = Cells_DelU[c][k];
}
void refh_get_rk_states(double *u1, double *u2) {
  for (int c = 0; c < No_Physical_Cells; c++)
    for (int k = 0; k < 4; k++) {
      u1[4 * c + k] = U_Cells_RK_1[c][k];
      u2[4 * c + k] = U_Cells_RK_2[c][k];
    }
}
void refh_get_dt(double *out) {
  for (int c = 0; c < No_Physical_Cells; c++) out[c] = Cells[c].del_t;
}
void refh_get_error(double *out) {
  for (int k = 0; k < 4; k++) out[k] = Error[k];
}
double refh_min_dt() { return Min_dt; }
double refh_total_time() { return Total_Time; }
int refh_iterations() { return iterations; }

// Individual entry points of the path.
void refh_apply_bc() { Apply_Boundary_Conditions(); }
// The residual the configured method evaluates: WENO when Is_WENO (Runge_Kutta_Method always;
// Explicit_Method only on all-quad meshes, src/Numerical_Method.cpp:31-55), else 1O / 2O.
void refh_net_flux() {
  quiet_begin();
  bool all_quads = true;
  for (int c = 0; c < No_Physical_Cells; c++) all_quads = all_quads && Cells[c].numFaces == 4;
  if (Is_WENO && (Time_Accurate || all_quads)) Evaluate_Cell_Net_Flux_WENO();
  else if (Is_Second_Order) Evaluate_Cell_Net_Flux_2O();
  else Evaluate_Cell_Net_Flux_1O();
  quiet_end();
}
double refh_get_min_dt() { return get_Min_dt(); }
// Net flux of every physical cell from zero through Calculate_Flux_For_All_Faces
// (src/Net_Flux.cpp:7-43) with the reference's ROE / ROE_2O as the dissipation callback.
void refh_net_flux_by_faces(double *out) {
  quiet_begin();
  for (int c = 0; c < No_Physical_Cells; c++) {
    for (int k = 0; k < 4; k++) Cells_Net_Flux[c][k] = 0.0;
    int cc = c;
    Calculate_Flux_For_All_Faces(cc, Is_Second_Order ? ROE_2O : ROE);
    for (int k = 0; k < 4; k++) out[4 * c + k] = Cells_Net_Flux[c][k];
  }
  quiet_end();
}
void refh_explicit() { quiet_begin(); Explicit_Method(); quiet_end(); }
void refh_lax_friedrichs() { Lax_Fedrichs(); }
void refh_rk3() { quiet_begin(); Runge_Kutta_Method(); quiet_end(); }
void refh_estimate_error() { Estimate_Error(); }
void refh_update() { Update(); }
// The reference's solution writers (src/output_files.cpp:492-556, src/Create_Vtk_File.cpp).
void refh_write_solution(const char *path) {
  Grid_Type = 0;
  nx_c = ny_c = nz_c = 0;
  Write_Solution(string(path), 1);
}
void refh_read_write_grid(const char *grid, const char *out) { Read_Write_Grid(string(grid), string(out)); }
void refh_append_solution(const char *sol, const char *out) {
  Grid_Type = 0;
  Append_Solution(string(sol), string(out));
}
void refh_ausm_net_flux() {
  for (int c = 0; c < No_Physical_Cells; c++) Ausm_Flux(c);
}
// The reference's fixed-pressure exit (src/Exit_Boundary_Conditions.cpp:8-66, which its
// Apply_Boundary_Conditions does not call) on every exit entry, from the current primitives.
void refh_exit_fixed_p() {
  for (unsigned int i = 0; i + 2 < Exit_Cells_List.size(); i += 3) Subsonic_Exit_Boundary_Condition(i);
}

// The loop body of Inviscid_Solver (src/Solver.cpp:94-125), n times or until t_end is reached
// (t_end <= 0: no time limit).  Returns the number of iterations performed.
int refh_iterate(int n, double t_end) {
  int done = 0;
  quiet_begin();
  for (int it = 0; it < n; it++) {
    Apply_Boundary_Conditions();
    if (Time_Accurate) Runge_Kutta_Method();
    else Explicit_Method();
    Total_Time += Min_dt;
    iterations++;
    Estimate_Error();
    Update();
    if (Enable_AMR && iterations > 0 && iterations % AMR_Period == 0) Apply_Adaptive_Refinement();
    done++;
    if (t_end > 0.0 && Total_Time >= t_end) break;
  }
  // With the B200 drop-in linked and lazy copies chosen, the globals the getters read are brought
  // up to date once here.
  if (b200_shim_sync) b200_shim_sync();
  quiet_end();
  return done;
}

// With the B200 drop-in linked: copy the device state into the globals after every entry point
// (k = 1, the default) or at every k-th Update() only.  Returns 0, or -1 without the drop-in.
int refh_set_shim_sync(int k) {
  if (!b200_shim_set_sync_every) return -1;
  b200_shim_set_sync_every(k);
  return 0;
}

// Green-Gauss gradient of primitive slot `var` (src/Grid_Refine_Functions.cpp:221-246).
void refh_gradient(int var, double *out) {
  V_D g(2, 0.0);
  for (int c = 0; c < No_Physical_Cells; c++) {
    int cc = c, vv = var;
    Calculate_Gradient_At_Cell_Center(cc, vv, g);
    out[2 * c] = g[0];
    out[2 * c + 1] = g[1];
  }
}

// AMR indicator and tags (src/Grid_Refine_Functions.cpp:8-63).
void refh_amr(double threshold, double max_fraction, double *indicator, unsigned char *tags) {
  AMR_Max_Fraction = max_fraction;
  double thr = threshold;
  TagRefinableCells(Cells, thr);
  for (int c = 0; c < No_Physical_Cells; c++) {
    indicator[c] = Gradient_Refinement_Indicator[c];
    tags[c] = Cells[c].Is_Splittable ? 1 : 0;
  }
}

// The reference's viscous residual on the current state: the set-up its Form_Cells does for a
// viscous wall (Construct_Co_Volumes per physical cell, src/Grid_Computations.cpp:367-375), the
// secondary neighbours of its face-gradient stencil (Identify_Neighbours_For_Second_Gradients,
// src/Grid_Refine_Functions.cpp:107-170), then Evaluate_Viscous_Fluxes
// (src/Grid_Refine_Functions.cpp:482-500) with Inv_Re and K1 set to the given nonzero values.
// flux: [NP][4] Cells_Viscous_Flux.  covol[0..2]: the largest |co-volume face area|, |co-volume
// face normal component| and |co-volume Inv_Area| over the cells.  stdout is left as it is: the
// reference reports a degenerate co-volume there and terminates the process (exit(0) in
// Evaluate_Cross_Product, src/Grid_Computations.cpp:834-844).
void refh_viscous_flux(double inv_re, double k1, double *flux, double *covol) {
  Co_Volume_Cells.clear();
  for (int c = 0; c < No_Physical_Cells; c++) {
    int cc = c;
    Identify_Neighbours_For_Second_Gradients(cc);
    Construct_Co_Volumes(cc);
  }
  Inv_Re = inv_re;
  K1 = k1;
  Evaluate_Viscous_Fluxes();
  covol[0] = covol[1] = covol[2] = 0.0;
  for (const Cell &C : Co_Volume_Cells) {
    for (double a : C.Face_Areas) covol[0] = std::max(covol[0], std::fabs(a));
    for (double n : C.Face_Normals) covol[1] = std::max(covol[1], std::fabs(n));
    covol[2] = std::max(covol[2], std::fabs(C.Inv_Area));
  }
  for (int c = 0; c < No_Physical_Cells; c++)
    for (int k = 0; k < 4; k++) flux[4 * c + k] = Cells_Viscous_Flux[c][k];
}

}  // extern "C"
