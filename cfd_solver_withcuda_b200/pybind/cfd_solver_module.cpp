// Python module CFD_Solver over the B200 C ABI: the scripting interface of the reference's
// pybind wrapper (Python_Wrapper/Euler_Python_Wrapper.cpp:92-159) for the explicit inviscid path,
// with the same function names, argument meaning and one process-wide solver like the reference's
// globals.  Every call goes through include/cfd_b200.h (libcfd_b200.so); the numerics run on the
// GPU.
//
// Kept from the reference module: readJSON, testCase, ReadGrid, FormCells, ConstructGhostCells,
// Inviscid_Solver, Explicit_Method, Runge_Kutta_Method, Evaluate_Time_Step, Inviscid_Time_Step,
// get_NoPhysical_Cells, get_Min_dt, get_Max_dt, Apply_Boundary_Conditions, Estimate_Error,
// Update, Set_DelU.  Added: Set_State and getters of the solution arrays as numpy arrays.
// Not provided (outside the explicit residual/update path): the implicit assembly (Assemble_A,
// Assemble_A1, Assemble_b, Compute_Flux_Jacobian, ComputeGhostCell_Flux_Jacobian and the index
// getters), Viscous_Solver and the viscous time steps, and the reference's cell-construction
// internals (ConstructCell, ConstructFace, ConstructCoVolumes, CheckCells, WriteCellInfo).
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <algorithm>
#include <fstream>
#include <iomanip>
#include <regex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "cfd_b200.h"

namespace py = pybind11;

namespace {

struct Solver {
  cfd_config cfg{};
  bool cfg_read = false;
  cfd_mesh *mesh = nullptr;
  cfd_mesh_desc desc{};
  cfd_ctx *ctx = nullptr;
  int total_iterations = 1000;
  double terminating_time = 0.0;
  bool time_dependent = false;
  int test_case = 0;
  std::vector<double> error = std::vector<double>(4, 0.0);
  double total_time = 0.0;
  int iterations = 0;
};

Solver &S() {
  static Solver s;
  return s;
}

void check(cfd_status st, const char *what) {
  if (st != CFD_OK) throw std::runtime_error(std::string(what) + ": " + cfd_last_error());
}

cfd_ctx *ctx() {
  Solver &s = S();
  if (!s.ctx) throw std::runtime_error("no solver: call ReadGrid and FormCells first");
  return s.ctx;
}

// Simulation keys the C ABI's config reader does not hold (src/Configuration_Read.cpp:23-87).
void read_simulation_keys(const std::string &path) {
  std::ifstream in(path);
  std::stringstream ss;
  ss << in.rdbuf();
  const std::string text = ss.str();
  std::smatch m;
  if (std::regex_search(text, m, std::regex("\"Total_Iterations\"\\s*:\\s*([0-9]+)")))
    S().total_iterations = std::stoi(m[1]);
  if (std::regex_search(text, m, std::regex("\"Terminating_Time\"\\s*:\\s*([-+0-9.eE]+)")))
    S().terminating_time = std::stod(m[1]);
  if (std::regex_search(text, m, std::regex("\"Is_Time_Dependent\"\\s*:\\s*(true|false|1|0)")))
    S().time_dependent = m[1] == "true" || m[1] == "1";
}

py::array_t<double> download(int which) {
  cfd_ctx *c = ctx();
  const Solver &s = S();
  const int NT = s.desc.n_physical + s.desc.n_ghost, NP = s.desc.n_physical;
  const int rows = which == 0 || which == 1 ? NT : NP;
  const int cols = which == 1 ? 11 : (which == 2 ? 1 : 4);
  py::array_t<double> out(std::vector<py::ssize_t>{rows, cols});
  double *p = out.mutable_data();
  check(cfd_download(c, which == 0 ? p : nullptr, which == 1 ? p : nullptr, which == 2 ? p : nullptr,
                     which == 3 ? p : nullptr, which == 4 ? p : nullptr),
        "download");
  return out;
}

void update_stats(const cfd_step_info &info) {
  Solver &s = S();
  for (int k = 0; k < 4; k++) s.error[k] = info.error[k];
  s.total_time = info.total_time;
  s.iterations = info.iterations;
}

}  // namespace

PYBIND11_MODULE(CFD_Solver, m) {
  m.doc() = "CFD solver on the B200: the reference wrapper's explicit inviscid interface over libcfd_b200";

  m.def("readJSON", [](const std::string &path) {
    Solver &s = S();
    cfd_config_default(&s.cfg);
    check(cfd_config_read_json(path.c_str(), &s.cfg), "readJSON");
    read_simulation_keys(path);
    s.cfg_read = true;
  }, py::arg("path"), "Reads a Solver_Config JSON file into the solver configuration");

  m.def("testCase", [](int test_case) { S().test_case = test_case; }, py::arg("Test_Case"),
        "Sets the test case ID (testCase 0 or any other: the initial state is the uniform inlet state of the "
        "configuration, or the one given to Set_State)");

  m.def("ReadGrid", [](const std::string &path) {
    Solver &s = S();
    if (s.mesh) cfd_mesh_destroy(s.mesh);
    s.mesh = nullptr;
    check(cfd_mesh_read_vtk(path.c_str(), &s.mesh), "ReadGrid");
    check(cfd_mesh_describe(s.mesh, &s.desc), "ReadGrid");
    return true;
  }, py::arg("path"), "Reads a legacy VTK grid (cells, faces, ghost cells and geometry as the reference's reader)");

  m.def("FormCells", []() {
    Solver &s = S();
    if (!s.mesh) throw std::runtime_error("FormCells: call ReadGrid first");
    if (!s.cfg_read) cfd_config_default(&s.cfg);
    if (s.ctx) cfd_destroy(s.ctx);
    s.ctx = nullptr;
    check(cfd_create(&s.desc, &s.cfg, &s.ctx), "FormCells");
    // Initial state: uniform inlet state (rho, u, v, p) of the configuration on every row.
    const int NT = s.desc.n_physical + s.desc.n_ghost;
    const double rho = s.cfg.inlet_rho, u = s.cfg.inlet_u, v = s.cfg.inlet_v, p = s.cfg.inlet_p;
    std::vector<double> U(4 * (size_t)NT);
    for (int c = 0; c < NT; c++) {
      U[4 * (size_t)c] = rho;
      U[4 * (size_t)c + 1] = rho * u;
      U[4 * (size_t)c + 2] = rho * v;
      U[4 * (size_t)c + 3] = (p / (1.4 - 1.0)) + rho * (0.5 * (u * u + v * v));
    }
    check(cfd_upload_state(s.ctx, U.data(), NT), "FormCells");
    s.iterations = 0;
    s.total_time = 0.0;
    return true;
  }, "Builds the GPU solver on the grid read by ReadGrid - returns True on success");

  m.def("ConstructGhostCells", []() {
    if (!S().mesh) throw std::runtime_error("ConstructGhostCells: call ReadGrid first");
  }, "Ghost cells are built by ReadGrid (the reference's Construct_Ghost_Cells numbering)");

  m.def("Set_State", [](py::array_t<double, py::array::c_style | py::array::forcecast> U) {
    if (U.ndim() != 2 || U.shape(1) != 4) throw std::runtime_error("Set_State: U must be [rows][4]");
    check(cfd_upload_state(ctx(), U.data(), static_cast<int>(U.shape(0))), "Set_State");
  }, py::arg("U"), "Conserved state rows U_Cells (physical, or physical + ghost) in reference order");

  m.def("Inviscid_Solver", [](const std::string &error_file, const std::string &solution_file) {
    Solver &s = S();
    cfd_ctx *c = ctx();
    std::ofstream err(error_file);
    if (!err) return false;
    err << std::setw(10) << "Iteration" << std::setw(15) << "Min_dt" << std::setw(15) << "Rho_Error" << std::setw(15)
        << "Rho_u_Error" << std::setw(15) << "Rho_v_Error" << std::setw(15) << "Rho_Et_Error" << std::setw(15)
        << "Total_Time" << "\n";
    const double t_end = s.time_dependent ? s.terminating_time : 0.0;
    const int header[3] = {s.test_case, s.cfg.dissipation_type, s.cfg.is_second_order};
    while (s.iterations < s.total_iterations) {
      const int chunk = std::min(1000 - s.iterations % 1000, s.total_iterations - s.iterations);
      cfd_step_info info{};
      const int before = s.iterations;
      if (cfd_step(c, chunk, t_end, &info) != CFD_OK) return false;
      update_stats(info);
      if (s.iterations <= before) break;  // t_end reached inside the chunk
      err << std::setw(10) << s.iterations << std::setw(15) << info.min_dt;
      for (int k = 0; k < 4; k++) err << std::setw(15) << s.error[k];
      err << std::setw(15) << s.total_time << "\n";
      if (cfd_write_solution(c, solution_file.c_str(), header, 3) != CFD_OK) return false;
      if (t_end > 0.0 && s.total_time >= t_end) break;
    }
    return true;
  }, py::arg("error_file"), py::arg("solution_file"),
     "Runs the inviscid loop (boundary conditions, explicit or Runge-Kutta update, Estimate_Error, Update) for "
     "Total_Iterations (or to Terminating_Time), writing the error history and the solution every 1000 "
     "iterations - returns True on success, False on failure");

  m.def("Explicit_Method", []() { check(cfd_explicit_method(ctx()), "Explicit_Method"); },
        "Executes the explicit method for solving");
  m.def("Runge_Kutta_Method", []() { check(cfd_runge_kutta_method(ctx()), "Runge_Kutta_Method"); },
        "Executes the Runge-Kutta method for solving");
  m.def("Apply_Boundary_Conditions", []() { check(cfd_apply_boundary_conditions(ctx()), "Apply_Boundary_Conditions"); },
        "Applies all boundary conditions based on the current setup");
  m.def("Estimate_Error", []() {
    double e[4];
    check(cfd_estimate_error(ctx(), e), "Estimate_Error");
    for (int k = 0; k < 4; k++) S().error[k] = e[k];
  }, "Estimates the error in a given iteration");
  m.def("Update", []() { check(cfd_update(ctx()), "Update"); }, "Updates the Solution vector");
  m.def("Set_DelU", [](py::array_t<double, py::array::c_style | py::array::forcecast> dU) {
    const Solver &s = S();
    if (dU.size() != 4 * (py::ssize_t)s.desc.n_physical) throw std::runtime_error("Set_DelU: need 4 * NP values");
    check(cfd_set_delu(ctx(), dU.data()), "Set_DelU");
  }, py::arg("dU"), "Sets the delU values for the cells");

  auto time_step = [](int cell) {
    cfd_ctx *c = ctx();
    const int NP = S().desc.n_physical;
    if (cell < 0 || cell >= NP) throw std::runtime_error("cell index out of range");
    check(cfd_evaluate_net_flux(c), "Evaluate_Time_Step");
    std::vector<double> dt(NP);
    check(cfd_download(c, nullptr, nullptr, dt.data(), nullptr, nullptr), "Evaluate_Time_Step");
    return dt[cell];
  };
  m.def("Evaluate_Time_Step", time_step, py::arg("cellIndex"),
        "Evaluates the time step (every cell's, on the GPU) and returns the given cell's");
  m.def("Inviscid_Time_Step", time_step, py::arg("cellIndex"), "Inviscid solver time step of a cell");

  m.def("get_NoPhysical_Cells", []() { return S().desc.n_physical; }, "Returns the number of physical cells");
  m.def("get_Min_dt", []() {
    double v = 0.0;
    check(cfd_get_min_dt(ctx(), &v), "get_Min_dt");
    return v;
  }, "Returns the minimum time step of all the cells");
  m.def("get_Max_dt", []() {
    const int NP = S().desc.n_physical;
    std::vector<double> dt(NP);
    check(cfd_download(ctx(), nullptr, nullptr, dt.data(), nullptr, nullptr), "get_Max_dt");
    double mx = 0.0;
    for (double d : dt) mx = std::max(mx, d);
    return mx;
  }, "Returns the maximum time step of all the cells");

  m.def("get_U", []() { return download(0); }, "U_Cells [NP+NG][4]");
  m.def("get_Primitive", []() { return download(1); }, "Primitive_Cells [NP+NG][11]");
  m.def("get_del_t", []() { return download(2); }, "Cell del_t [NP][1]");
  m.def("get_Net_Flux", []() { return download(3); }, "Cells_Net_Flux [NP][4]");
  m.def("get_DelU", []() { return download(4); }, "Cells_DelU [NP][4]");
  m.def("get_Error", []() { return S().error; }, "Error[4] of the last Estimate_Error or Inviscid_Solver chunk");
  m.def("reset", []() {
    Solver &s = S();
    if (s.ctx) cfd_destroy(s.ctx);
    if (s.mesh) cfd_mesh_destroy(s.mesh);
    s.ctx = nullptr;
    s.mesh = nullptr;
  }, "Releases the solver and the grid");
}
