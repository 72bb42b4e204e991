// Host-side mesh layer: generators, legacy-VTK I/O and the reference's mesh ingest rules.
//
// The arrays produced here are the reference's per-cell `Cell` data (include/Globals.h:313-328)
// in the reference's own ordering, so the CUDA path sees exactly the geometry and connectivity
// the reference would build from the same points and cells.
#pragma once
#include <cstdint>
#include <map>
#include <string>
#include <utility>
#include <vector>

namespace cfdb {

enum BoundaryKind : int { BK_INLET = 0, BK_EXIT = 1, BK_WALL = 2, BK_SYMMETRY = 3 };

struct Mesh {
  // Raw input: points (x, y, z) and cells as node lists (3 or 4 nodes).
  std::vector<double> points;
  std::vector<std::vector<int>> cell_nodes;
  // Optional boundary kinds keyed by the sorted node pair of a boundary edge.  When empty the
  // reference's bounding-box classification is used (src/Read_Gmsh_File.cpp:490-625).
  std::map<std::pair<int, int>, int> edge_kind;

  // Derived, reference order (filled by build()).
  int n_physical = 0;
  int n_ghost = 0;
  std::vector<int> n_faces;          // [NP]
  std::vector<int> nodes_sorted;     // [NP*4] anticlockwise node order, -1 padded
  std::vector<int> nbr;              // [NP*4] neighbour or ghost id, -1 padded
  std::vector<double> normals;       // [NP*8]
  std::vector<double> lengths;       // [NP*4]
  std::vector<double> ccd;           // [NP*4] centre-to-centre distances
  std::vector<double> cvec;          // [NP*8] centre-to-centre vectors (x, y) per face
  std::vector<double> area;          // [NP]
  std::vector<double> inv_area;      // [NP]
  std::vector<double> centers;       // [(NP+NG)*3]
  std::vector<int> boundary;         // [NB*4]: kind, cell, face, ghost (list order: inlet, exit, wall, symmetry)
  std::vector<int> lists[4];         // per-kind triples (cell, face, ghost) in reference list order

  std::string build();               // returns "" on success, else an error message
};

// Generators.  All return "" on success.
std::string generate_box(Mesh &m, int nx, int ny, double x0, double x1, double y0, double y1);
std::string generate_half_cylinder(Mesh &m, int ntheta, int nr, double r_body, double r_outer, double ratio);
std::string generate_ramp(Mesh &m, int nx, int ny, double length, double height, double x_corner, double angle_deg,
                          int open_top);
std::string generate_bump(Mesh &m, int nx, int ny, double length, double height, double thickness, int n_quad_layers,
                          double jitter, uint64_t seed, int triangles);

std::string read_vtk(Mesh &m, const std::string &path);
std::string write_vtk(const Mesh &m, const std::string &path);

// Reverse Cuthill-McKee order of the physical cells (perm[new] = old).

}  // namespace cfdb
