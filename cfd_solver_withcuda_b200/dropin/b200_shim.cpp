// Drop-in translation unit for the reference solver (rameshkolluru43/CFD_Solver_withCUDA).
//
// Link this file in place of the reference's src/Numerical_Method.cpp, src/Net_Flux.cpp,
// src/Error_Estimate_Update.cpp and src/Boundary_Conditions.cpp, and link libcfd_b200.so: the
// reference's own driver then runs its boundary-condition, residual and update path on the GPU.  It implements the same entry points with the same
// signatures over the reference's globals (include/Globals.h:332-416) and, like the reference,
// exits on errors.  Compiled against the reference's headers; it is not part of libcfd_b200.so.
//
// Post-conditions (e.g. after Runge_Kutta_Method: Cells_DelU = dU, Primitive_Cells = stage-2
// primitives, U_Cells unchanged, Min_dt set) are met by copying the device state back into the
// globals.  By default that happens after every entry point, so every global is what the
// reference would hold.  A driver whose loop reads only Min_dt and Error between its output steps
// can make the copies lazy: b200_shim_set_sync_every(k) (or CFD_B200_SYNC_EVERY=k in the
// environment) copies the state back at every k-th Update() only (k = 0: never by itself), and
// b200_shim_sync() copies it at once, e.g. before Write_Solution.  Min_dt and Error are always
// set after each call.
#include "definitions.h"
#include "Globals.h"
#include "Flux.h"
#include "Primitive_Computational.h"
#include "cfd_b200.h"

#include <algorithm>
#include <cstdlib>

V_D Error(4, 0.0);  // src/Error_Estimate_Update.cpp:7

namespace {
cfd_ctx *g_ctx = nullptr;
int g_sync_every = -1;   // -1: not yet read from the environment; 1: eager; k > 1: every k-th Update(); 0: on request
long long g_updates = 0;
bool g_dirty = false;    // the device holds state the globals do not
std::vector<int> g_nf, g_nbr, g_bnd;
std::vector<double> g_nrm, g_len, g_ccd, g_cvec, g_area, g_inva;

void b200_check(cfd_status s) {
  if (s != CFD_OK) {
    fprintf(stderr, "cfd_b200: %s\n", cfd_last_error());
    exit(EXIT_FAILURE);
  }
}

// Mesh, configuration and state from the reference's globals, on first use.
void b200_init() {
  const int NP = No_Physical_Cells;
  g_nf.assign(NP, 0);
  g_nbr.assign(4 * (size_t)NP, -1);
  g_nrm.assign(8 * (size_t)NP, 0.0);
  g_len.assign(4 * (size_t)NP, 0.0);
  g_ccd.assign(4 * (size_t)NP, 0.0);
  g_cvec.assign(8 * (size_t)NP, 0.0);
  g_area.assign(NP, 0.0);
  g_inva.assign(NP, 0.0);
  for (int c = 0; c < NP; c++) {
    const Cell &C = Cells[c];
    g_nf[c] = C.numFaces;
    g_area[c] = C.Area;
    g_inva[c] = C.Inv_Area;
    for (int f = 0; f < C.numFaces; f++) {
      g_nbr[4 * c + f] = C.Neighbours[f];
      g_len[4 * c + f] = C.Face_Areas[f];
      g_nrm[8 * c + 2 * f] = C.Face_Normals[2 * f];
      g_nrm[8 * c + 2 * f + 1] = C.Face_Normals[2 * f + 1];
      g_ccd[4 * c + f] = C.Cell_Center_Distances[f];
      if (C.Cell_Center_Vector.size() >= 3 * (size_t)(f + 1)) {
        g_cvec[8 * c + 2 * f] = C.Cell_Center_Vector[3 * f];
        g_cvec[8 * c + 2 * f + 1] = C.Cell_Center_Vector[3 * f + 1];
      }
    }
  }
  g_bnd.clear();
  auto add = [](int kind, const V_I &l) {
    for (size_t i = 0; i + 2 < l.size(); i += 3) g_bnd.insert(g_bnd.end(), {kind, l[i], l[i + 1], l[i + 2]});
  };
  add(CFD_BC_INLET, Inlet_Cells_List);
  add(CFD_BC_EXIT, Exit_Cells_List);
  add(CFD_BC_WALL, Wall_Cells_List);
  if (has_Symmetry_BC) add(CFD_BC_SYMMETRY, Symmetry_Cells_List);
  cfd_mesh_desc d = {NP,          No_Ghost_Cells, g_nf.data(),   g_nbr.data(),  g_nrm.data(),
                     g_len.data(), g_ccd.data(),  g_cvec.data(), g_area.data(), g_inva.data(),
                     static_cast<int>(g_bnd.size() / 4), g_bnd.data()};
  cfd_config cfg;
  cfd_config_default(&cfg);
  cfg.dissipation_type = Dissipation_Type;
  cfg.movers_single_alpha = Is_MOVERS_1 ? 1 : 0;
  cfg.movers_entropy_fix = Enable_Entropy_Fix ? 1 : 0;
  cfg.is_second_order = Is_Second_Order ? 1 : 0;
  cfg.time_accurate = Time_Accurate ? 1 : 0;
  cfg.local_time_stepping = Local_Time_Stepping ? 1 : 0;
  cfg.cfl = CFL;
  cfg.limiter_zeta = Limiter_Zeta;
  cfg.limiter_zeta1 = Limiter_Zeta1;
  cfg.weno = Is_WENO ? 1 : 0;
  cfg.weno_characteristic = Is_Char ? 1 : 0;
  cfg.inlet_bc = Is_Inlet_SubSonic ? CFD_INLET_SUBSONIC_REF : CFD_INLET_SUPERSONIC;
  cfg.exit_bc = Is_Exit_SubSonic ? CFD_EXIT_SUBSONIC_REF : CFD_EXIT_SUPERSONIC;
  cfg.inlet_rho = inletCond.Rho;
  cfg.inlet_p = inletCond.P;
  b200_check(cfd_create(&d, &cfg, &g_ctx));
  std::vector<double> U(4 * (size_t)Total_No_Cells);
  for (int c = 0; c < Total_No_Cells; c++)
    for (int k = 0; k < 4; k++) U[4 * (size_t)c + k] = U_Cells[c][k];
  b200_check(cfd_upload_state(g_ctx, U.data(), Total_No_Cells));
}

void ensure() {
  if (g_sync_every < 0) {
    const char *e = std::getenv("CFD_B200_SYNC_EVERY");
    g_sync_every = e ? std::max(0, std::atoi(e)) : 1;
  }
  if (!g_ctx) b200_init();
}

// Device state -> the reference's globals.
void sync_globals() {
  const int NT = Total_No_Cells, NP = No_Physical_Cells;
  std::vector<double> U(4 * (size_t)NT), P(11 * (size_t)NT), dt(NP), net(4 * (size_t)NP), dU(4 * (size_t)NP);
  b200_check(cfd_download(g_ctx, U.data(), P.data(), dt.data(), net.data(), dU.data()));
  for (int c = 0; c < NT; c++) {
    for (int k = 0; k < 4; k++) U_Cells[c][k] = U[4 * (size_t)c + k];
    for (int k = 0; k < 11; k++) Primitive_Cells[c][k] = P[11 * (size_t)c + k];
  }
  for (int c = 0; c < NP; c++) {
    Cells[c].del_t = dt[c];
    for (int k = 0; k < 4; k++) {
      Cells_Net_Flux[c][k] = net[4 * (size_t)c + k];
      Cells_DelU[c][k] = dU[4 * (size_t)c + k];
    }
  }
  b200_check(cfd_get_min_dt(g_ctx, &Min_dt));
  g_dirty = false;
}

// After an entry point that changed the device state: Min_dt at once, the rest by the sync rule.
void changed(bool is_update) {
  b200_check(cfd_get_min_dt(g_ctx, &Min_dt));
  g_dirty = true;
  if (is_update) g_updates++;
  if (g_sync_every == 1 || (is_update && g_sync_every > 1 && g_updates % g_sync_every == 0)) sync_globals();
}
}  // namespace

// Copies the device state into the reference's globals now (a no-op when they are current).
extern "C" void b200_shim_sync() {
  if (g_ctx && g_dirty) sync_globals();
}

// k = 1 (default): copy after every entry point; k > 1: at every k-th Update(); k = 0: only on
// b200_shim_sync().
extern "C" void b200_shim_set_sync_every(int k) {
  b200_shim_sync();
  g_sync_every = k < 0 ? 0 : k;
}

// Releases the device context (the next entry point re-reads mesh, configuration and state from
// the globals); for drivers that load a new mesh into the same process.
extern "C" void b200_shim_reset() {
  if (g_ctx) cfd_destroy(g_ctx);
  g_ctx = nullptr;
  g_dirty = false;
  g_updates = 0;
}

// src/Boundary_Conditions.cpp:12-61: the ghost rows of every boundary entry, on the device.
void Apply_Boundary_Conditions() {
  ensure();
  b200_check(cfd_apply_boundary_conditions(g_ctx));
  changed(false);
}

// src/Net_Flux.cpp:46,97 — both orders: the context was configured from Is_Second_Order.
void Evaluate_Cell_Net_Flux_1O() {
  ensure();
  b200_check(cfd_evaluate_net_flux(g_ctx));
  changed(false);
}
void Evaluate_Cell_Net_Flux_2O() { Evaluate_Cell_Net_Flux_1O(); }

// src/Numerical_Method.cpp:322 — Min_dt of the last flux evaluation.
double get_Min_dt() {
  ensure();
  b200_check(cfd_get_min_dt(g_ctx, &Min_dt));
  return Min_dt;
}
double get_Max_dt() {
  b200_shim_sync();
  double m = 0.0;
  for (int c = 0; c < No_Physical_Cells; c++) m = std::max(m, Cells[c].del_t);
  Max_dt = m;
  return Max_dt;
}

// src/Numerical_Method.cpp:26 / :342.  The boundary conditions are applied on the device first,
// as the driver's Apply_Boundary_Conditions just did (same values), so that a driver that changed
// nothing in between and one that calls the method alone get the same result.
void Explicit_Method() {
  ensure();
  b200_check(cfd_apply_boundary_conditions(g_ctx));
  cfd_status s = cfd_explicit_method(g_ctx);
  if (s == CFD_ERR_DT_NONPOSITIVE) {
    fprintf(stderr, "Error: Min_dt is zero. Cannot proceed with the simulation.\n");
    exit(EXIT_FAILURE);
  }
  b200_check(s);
  changed(false);
}
void Runge_Kutta_Method() {
  ensure();
  b200_check(cfd_apply_boundary_conditions(g_ctx));
  b200_check(cfd_runge_kutta_method(g_ctx));
  changed(false);
}
void Implicit_Method() { fprintf(stderr, "Implicit_Method is not part of the B200 path.\n"); }
// src/Numerical_Method.cpp:459.
void Lax_Fedrichs() {
  ensure();
  b200_check(cfd_lax_friedrichs(g_ctx));
  changed(false);
}

// src/Error_Estimate_Update.cpp:10 / :31.
void Estimate_Error() {
  ensure();
  double e[4];
  b200_check(cfd_estimate_error(g_ctx, e));
  for (int k = 0; k < 4; k++) Error[k] = e[k];
}
void Update() {
  ensure();
  b200_check(cfd_update(g_ctx));
  changed(true);
}

// src/Net_Flux.cpp:7-43: adds the average flux minus the given dissipation of every face of one
// cell to Cells_Net_Flux.  The dissipation is a host function by its signature (ROE, LLF, ... of
// the reference), so this helper runs on the host over the globals, brought up to date first; the
// solver's own net-flux entry points above do not use it.
void Calculate_Flux_For_All_Faces(int &Current_Cell_No, void (*Dissipation_Function)(const int &, int &, const int &)) {
  b200_shim_sync();
  const Cell &C = Cells[Current_Cell_No];
  const int n_faces = C.numFaces > 0 ? C.numFaces : static_cast<int>(C.Face_Areas.size());
  const int n_nbr = static_cast<int>(C.Neighbours.size());
  for (int face = 0; face < n_faces && face < n_nbr; face++) {
    int nb = C.Neighbours[face];
    if (nb < 0) continue;
    const bool on_boundary = Current_Cell_No < static_cast<int>(Cells_Face_Boundary_Type.size()) &&
                             face < static_cast<int>(Cells_Face_Boundary_Type[Current_Cell_No].size()) &&
                             Cells_Face_Boundary_Type[Current_Cell_No][face];
    Calculate_Face_Average_Flux(Current_Cell_No, nb, face, on_boundary);
    Dissipation_Function(Current_Cell_No, nb, face);
    for (int v = 0; v < NUM_FLUX_COMPONENTS; v++)
      Cells_Net_Flux[Current_Cell_No][v] += Average_Convective_Flux[v] - Dissipative_Flux[v];
  }
}

// Per-cell primitive refreshes of src/Error_Estimate_Update.cpp:46-77, still used by other
// reference files: host EOS on the given row, as the reference does.
void Update(int &Cell_Index, int &Update_Type) {
  Calculate_Primitive_Variables(Cell_Index, Update_Type == 1 ? U_Cells_RK_1[Cell_Index] : U_Cells_RK_2[Cell_Index]);
  Primitive_Cells[Cell_Index] = Global_Primitive;
}
void Update(const int &Cell_Index, V_D &U) {
  Calculate_Primitive_Variables(Cell_Index, U);
  Primitive_Cells[Cell_Index] = Global_Primitive;
}
void Update(const int &Cell_Index) {
  Calculate_Primitive_Variables(Cell_Index, U_Cells[Cell_Index]);
  Primitive_Cells[Cell_Index] = Global_Primitive;
}
