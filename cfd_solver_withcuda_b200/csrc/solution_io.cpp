// Solution files on either side of the path, in the reference's on-disk formats (host only).
//
//   cfd_vtk_copy_grid        Read_Write_Grid, src/Create_Vtk_File.cpp:5-53
//   cfd_vtk_append_solution  Append_Solution, src/Create_Vtk_File.cpp:55-157
//
// Both are written with the same stream operations as the reference (default stream precision,
// the same separators), so the files are byte-identical to the reference's for the same inputs.
// Like the reference, the appended cell data is read back from the solution text file (values
// at six significant digits), and the entropy column is formed from those read-back values.
#include <cmath>
#include <fstream>
#include <string>
#include <vector>

#include "cfd_b200.h"

namespace cfdb {
void set_last_error(const std::string &msg);
}

extern "C" {

cfd_status cfd_vtk_copy_grid(const char *grid_vtk, const char *out_vtk) {
  if (!grid_vtk || !out_vtk) {
    cfdb::set_last_error("cfd_vtk_copy_grid: null path");
    return CFD_ERR_BAD_ARG;
  }
  std::ifstream in(grid_vtk);
  if (!in.is_open()) {
    cfdb::set_last_error(std::string("cannot open ") + grid_vtk);
    return CFD_ERR_IO;
  }
  std::ofstream out(out_vtk);
  if (!out.is_open()) {
    cfdb::set_last_error(std::string("cannot write ") + out_vtk);
    return CFD_ERR_IO;
  }
  std::string s1, s2;
  for (int k = 0; k < 4; k++) {
    std::getline(in, s1);
    out << s1 << std::endl;
  }
  int nop = 0, n_cells = 0;
  in >> s1 >> nop >> s2;
  out << s1 << "\t" << nop << "\t" << s2 << std::endl;
  for (int i = 0; i < nop; i++) {
    double x, y, z;
    in >> x >> y >> z;
    out << x << "\t" << y << "\t" << z << std::endl;
  }
  in >> s1 >> n_cells >> nop;
  out << s1 << "\t" << n_cells << "\t" << nop << std::endl;
  for (int i = 0; i < n_cells; i++) {
    long a, b, c, d, e;
    in >> a >> b >> c >> d >> e;
    out << a << "\t" << b << "\t" << c << "\t" << d << "\t" << e << std::endl;
  }
  in >> s1 >> nop;
  out << s1 << "\t" << nop << std::endl;
  for (int i = 0; i < nop; i++) {
    int p;
    in >> p;
    out << p << std::endl;
  }
  return CFD_OK;
}

cfd_status cfd_vtk_append_solution(const char *solution_txt, const char *out_vtk, int n_header) {
  if (!solution_txt || !out_vtk || n_header < 0) {
    cfdb::set_last_error("cfd_vtk_append_solution: bad argument");
    return CFD_ERR_BAD_ARG;
  }
  std::ifstream in(solution_txt);
  if (!in.is_open()) {
    cfdb::set_last_error(std::string("cannot open ") + solution_txt);
    return CFD_ERR_IO;
  }
  std::ofstream out(out_vtk, std::ios::out | std::ios::app);
  if (!out.is_open()) {
    cfdb::set_last_error(std::string("cannot write ") + out_vtk);
    return CFD_ERR_IO;
  }
  for (int k = 0; k < n_header; k++) {
    int h;
    in >> h;
  }
  int n_cells = 0, iterations = 0;
  in >> n_cells >> iterations;
  std::vector<double> P, T, Rho, U, V, M, P0;
  for (int i = 0; i < n_cells; i++) {
    int idx;
    double dt, rho, p, t, u, v, mach, p0;
    in >> idx >> dt >> rho >> p >> t >> u >> v >> mach >> p0;
    P.push_back(p);
    Rho.push_back(rho);
    T.push_back(t);
    U.push_back(u);
    V.push_back(v);
    M.push_back(mach);
    P0.push_back(p0);
  }
  auto scalars = [&](const char *head, const std::vector<double> &x) {
    out << head << std::endl;
    out << "LOOKUP_TABLE default" << std::endl;
    for (double w : x) out << w << std::endl;
  };
  out << "CELL_DATA\t" << n_cells << std::endl;
  scalars("SCALARS\t Pressure\t double", P);
  scalars("SCALARS\t Temperature\t double ", T);
  scalars("SCALARS\t Density\t double ", Rho);
  scalars("SCALARS\t U_Velocity\t double ", U);
  scalars("SCALARS\t V_Velocity\t double", V);
  scalars("SCALARS\t Total_Pressure\t double", P0);
  out << "SCALARS\t Entropy\t double" << std::endl;
  out << "LOOKUP_TABLE default" << std::endl;
  for (size_t i = 0; i < P.size(); i++) out << std::log(P[i] / std::pow(Rho[i], 1.4)) << std::endl;
  scalars("SCALARS\t Mach_Number\t double ", M);
  out << "Vectors\t Velocity\t double " << std::endl;
  for (int i = 0; i < n_cells; i++) out << U[i] << "\t" << V[i] << "\t" << 0.0 << std::endl;
  return CFD_OK;
}

}  // extern "C"
