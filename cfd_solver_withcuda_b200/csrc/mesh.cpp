// Host-side mesh layer (see mesh.hpp).
//
// build() restates the reference's mesh ingest so that geometry and connectivity are
// bit-identical to what the reference computes from the same points:
//   anticlockwise vertex sort        src/Grid_Computations.cpp:1092-1139 (+ :957-979, :1021-1035)
//   centroid / faces / shoelace area src/Grid_Computations.cpp:523-565, :691-752
//   face-ordered neighbours, ghosts  src/Read_Gmsh_File.cpp:325-402 (ghost ids cell-major, face-minor)
//   bounding-box classification      src/Read_Gmsh_File.cpp:441-472, :490-625
//   ghost centres                    src/Grid_Computations.cpp:394-442, :589-629
//   centre distances                 src/Grid_Computations.cpp:802-827, :863-888
#include "mesh.hpp"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <queue>
#include <set>
#include <sstream>

namespace cfdb {

namespace {

constexpr double kEpsilon = 1e-6;  // EPSILON, include/definitions.h:70
constexpr int FK_INTERNAL = 0, FK_LEFT = 1, FK_RIGHT = 2, FK_TOP = 3, FK_BOTTOM = 4, FK_WALL = 5;

using P3 = std::array<double, 3>;

// Vertex average, summed in list order and divided by the integer count.
P3 centroid_of(const std::vector<P3> &v) {
  double x = 0.0, y = 0.0, z = 0.0;
  int n = static_cast<int>(v.size());
  for (const P3 &p : v) {
    x += p[0];
    y += p[1];
    z += p[2];
  }
  P3 c{0.0, 0.0, 0.0};
  if (n > 0) {
    c[0] = x / n;
    c[1] = y / n;
    c[2] = z / n;
  }
  return c;
}

// Sorts (vertex, node) pairs by polar angle about the vertex average unless they are already
// in non-decreasing angle order; ties within 1e-9 rad are broken by z.
void sort_anticlockwise(std::vector<P3> &verts, std::vector<int> &nodes) {
  P3 c = centroid_of(verts);
  std::vector<std::pair<P3, int>> pr;
  for (size_t i = 0; i < verts.size(); i++) pr.emplace_back(verts[i], nodes[i]);
  bool sorted = true;
  for (size_t i = 1; i < pr.size(); ++i) {
    double a0 = std::atan2(pr[i - 1].first[1] - c[1], pr[i - 1].first[0] - c[0]);
    double a1 = std::atan2(pr[i].first[1] - c[1], pr[i].first[0] - c[0]);
    if (a0 > a1) {
      sorted = false;
      break;
    }
  }
  if (!sorted) {
    std::sort(pr.begin(), pr.end(), [&c](const std::pair<P3, int> &a, const std::pair<P3, int> &b) {
      double angleA = std::atan2(a.first[1] - c[1], a.first[0] - c[0]);
      double angleB = std::atan2(b.first[1] - c[1], b.first[0] - c[0]);
      if (std::abs(angleA - angleB) < 1e-9) return a.first[2] < b.first[2];
      return angleA < angleB;
    });
  }
  for (size_t i = 0; i < pr.size(); i++) {
    verts[i] = pr[i].first;
    nodes[i] = pr[i].second;
  }
}

int classify_edge(const P3 &p1, const P3 &p2, double minX, double maxX, double minY, double maxY) {
  if (std::abs(p1[0] - minX) < kEpsilon && std::abs(p2[0] - minX) < kEpsilon) return FK_LEFT;
  if (std::abs(p1[0] - maxX) < kEpsilon && std::abs(p2[0] - maxX) < kEpsilon) return FK_RIGHT;
  if (std::abs(p1[1] - minY) < kEpsilon && std::abs(p2[1] - minY) < kEpsilon) return FK_BOTTOM;
  if (std::abs(p1[1] - maxY) < kEpsilon && std::abs(p2[1] - maxY) < kEpsilon) return FK_TOP;
  return FK_WALL;
}

std::pair<int, int> edge_key(int a, int b) { return a < b ? std::make_pair(a, b) : std::make_pair(b, a); }

}  // namespace

std::string Mesh::build() {
  const int NP = static_cast<int>(cell_nodes.size());
  if (NP == 0) return "mesh has no cells";
  const int npts = static_cast<int>(points.size() / 3);
  n_physical = NP;
  n_faces.assign(NP, 0);
  nodes_sorted.assign(static_cast<size_t>(NP) * 4, -1);
  normals.assign(static_cast<size_t>(NP) * 8, 0.0);
  lengths.assign(static_cast<size_t>(NP) * 4, 0.0);
  ccd.assign(static_cast<size_t>(NP) * 4, 0.0);
  area.assign(NP, 0.0);
  inv_area.assign(NP, 0.0);
  std::vector<std::vector<P3>> cverts(NP);
  std::vector<P3> ccent(NP);

  for (int i = 0; i < NP; i++) {
    std::vector<int> nodes = cell_nodes[i];
    const int n = static_cast<int>(nodes.size());
    if (n != 3 && n != 4) return "cell " + std::to_string(i) + " is not a triangle or quadrilateral";
    std::vector<P3> v(n);
    for (int k = 0; k < n; k++) {
      int p = nodes[k];
      if (p < 0 || p >= npts) return "cell " + std::to_string(i) + " references a missing point";
      v[k] = P3{points[3 * p], points[3 * p + 1], points[3 * p + 2]};
    }
    sort_anticlockwise(v, nodes);
    n_faces[i] = n;
    for (int k = 0; k < n; k++) nodes_sorted[4 * i + k] = nodes[k];
    ccent[i] = centroid_of(v);
    for (int f = 0; f < n; f++) {
      const P3 &a = v[f];
      const P3 &b = v[(f + 1) % n];
      double dy = b[1] - a[1];
      double dx = b[0] - a[0];
      double dL = std::sqrt(dx * dx + dy * dy);
      if (dL == 0.0) return "cell " + std::to_string(i) + " has a zero-length face";
      lengths[4 * i + f] = dL;
      normals[8 * i + 2 * f] = dy / dL;
      normals[8 * i + 2 * f + 1] = -dx / dL;
    }
    double twice_area = 0.0;
    for (int k = 0; k < n; k++) {
      int j = (k + 1) % n;
      twice_area += (v[k][0] * v[j][1] - v[j][0] * v[k][1]);
    }
    area[i] = 0.5 * std::fabs(twice_area);
    if (!std::isfinite(area[i]) || area[i] <= 0.0) return "cell " + std::to_string(i) + " has a non-positive area";
    inv_area[i] = 1.0 / area[i];
    cverts[i] = std::move(v);
  }

  // Edge -> cells map over the sorted node lists, then face-ordered neighbours and ghost ids.
  std::map<std::pair<int, int>, std::set<int>> e2c;
  for (int i = 0; i < NP; i++) {
    int n = n_faces[i];
    for (int f = 0; f < n; f++) e2c[edge_key(nodes_sorted[4 * i + f], nodes_sorted[4 * i + (f + 1) % n])].insert(i);
  }
  nbr.assign(static_cast<size_t>(NP) * 4, -1);
  int ghost = NP;
  std::vector<char> has_boundary(NP, 0);
  for (int i = 0; i < NP; i++) {
    int n = n_faces[i];
    for (int f = 0; f < n; f++) {
      auto it = e2c.find(edge_key(nodes_sorted[4 * i + f], nodes_sorted[4 * i + (f + 1) % n]));
      if (it != e2c.end() && it->second.size() == 2) {
        for (int other : it->second)
          if (other != i) {
            nbr[4 * i + f] = other;
            break;
          }
      }
    }
    for (int f = 0; f < n; f++)
      if (nbr[4 * i + f] < 0) {
        nbr[4 * i + f] = ghost++;
        has_boundary[i] = 1;
      }
  }
  n_ghost = ghost - NP;

  // Boundary lists.
  for (auto &l : lists) l.clear();
  if (edge_kind.empty()) {
    double Xmin = 0, Xmax = 0, Ymin = 0, Ymax = 0;
    for (int p = 0; p < npts; p++) {
      double x = points[3 * p], y = points[3 * p + 1];
      if (p == 0) {
        Xmin = Xmax = x;
        Ymin = Ymax = y;
      } else {
        if (x < Xmin) Xmin = x;
        if (x > Xmax) Xmax = x;
        if (y < Ymin) Ymin = y;
        if (y > Ymax) Ymax = y;
      }
    }
    for (int i = 0; i < NP; i++) {
      int n = n_faces[i];
      for (int f = 0; f < n; f++) {
        int nb = nbr[4 * i + f];
        if (nb < NP) continue;
        int fk = has_boundary[i] ? classify_edge(cverts[i][f], cverts[i][(f + 1) % n], Xmin, Xmax, Ymin, Ymax) : FK_INTERNAL;
        int kind = fk == FK_LEFT ? BK_INLET : fk == FK_RIGHT ? BK_EXIT : (fk == FK_TOP || fk == FK_BOTTOM || fk == FK_WALL) ? BK_WALL : -1;
        if (kind < 0) continue;
        lists[kind].insert(lists[kind].end(), {i, f, nb});
      }
    }
  } else {
    for (int i = 0; i < NP; i++) {
      int n = n_faces[i];
      for (int f = 0; f < n; f++) {
        int nb = nbr[4 * i + f];
        if (nb < NP) continue;
        auto it = edge_kind.find(edge_key(nodes_sorted[4 * i + f], nodes_sorted[4 * i + (f + 1) % n]));
        if (it == edge_kind.end()) return "boundary edge of cell " + std::to_string(i) + " has no boundary kind";
        lists[it->second].insert(lists[it->second].end(), {i, f, nb});
      }
    }
  }
  boundary.clear();
  for (int k = 0; k < 4; k++)
    for (size_t e = 0; e < lists[k].size(); e += 3)
      boundary.insert(boundary.end(), {k, lists[k][e], lists[k][e + 1], lists[k][e + 2]});
  if (static_cast<int>(boundary.size() / 4) != n_ghost) return "some boundary faces were not classified";

  // Cell centres incl. ghosts mirrored through the face midpoint (inlet, wall, exit, symmetry).
  centers.assign(static_cast<size_t>(NP + n_ghost) * 3, 0.0);
  for (int i = 0; i < NP; i++)
    for (int k = 0; k < 3; k++) centers[3 * i + k] = ccent[i][k];
  const int order[4] = {BK_INLET, BK_WALL, BK_EXIT, BK_SYMMETRY};
  for (int kk : order) {
    const std::vector<int> &l = lists[kk];
    for (size_t e = 0; e < l.size(); e += 3) {
      int c = l[e], f = l[e + 1], g = l[e + 2];
      int nv = static_cast<int>(cverts[c].size());
      int i0 = f % nv, i1 = (f + 1) % nv;
      for (int k = 0; k < 3; k++) {
        double mid = 0.5 * (cverts[c][i0][k] + cverts[c][i1][k]);
        centers[3 * g + k] = ccent[c][k] + 2.0 * (mid - ccent[c][k]);
      }
    }
  }
  cvec.assign(static_cast<size_t>(NP) * 8, 0.0);
  for (int i = 0; i < NP; i++) {
    for (int f = 0; f < n_faces[i]; f++) {
      int N = nbr[4 * i + f];
      cvec[8 * i + 2 * f] = centers[3 * N] - centers[3 * i];
      cvec[8 * i + 2 * f + 1] = centers[3 * N + 1] - centers[3 * i + 1];
      double D = 0.0;
      for (int k = 0; k < 3; k++) {
        double t = centers[3 * N + k] - centers[3 * i + k];
        D += t * t;
      }
      ccd[4 * i + f] = std::sqrt(D);
    }
  }
  return "";
}

// ---------------------------------------------------------------------------------------------
// Generators
// ---------------------------------------------------------------------------------------------

std::string generate_box(Mesh &m, int nx, int ny, double x0, double x1, double y0, double y1) {
  if (nx < 1 || ny < 1) return "box needs nx, ny >= 1";
  m = Mesh();
  m.points.reserve(static_cast<size_t>(nx + 1) * (ny + 1) * 3);
  for (int j = 0; j <= ny; j++)
    for (int i = 0; i <= nx; i++) {
      m.points.push_back(x0 + (x1 - x0) * (static_cast<double>(i) / nx));
      m.points.push_back(y0 + (y1 - y0) * (static_cast<double>(j) / ny));
      m.points.push_back(0.0);
    }
  auto P = [nx](int i, int j) { return j * (nx + 1) + i; };
  m.cell_nodes.reserve(static_cast<size_t>(nx) * ny);
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) m.cell_nodes.push_back({P(i, j), P(i + 1, j), P(i + 1, j + 1), P(i, j + 1)});
  return "";  // bounding-box classification: left inlet, right exit, bottom/top wall
}

// Front half of a cylinder (theta in [pi/2, 3pi/2], facing -x) on a body-fitted O-grid with
// geometric radial stretching.  Body = slip wall, outer arc = supersonic inflow, the two radial
// cut lines on x = 0 = extrapolation outflow.
std::string generate_half_cylinder(Mesh &m, int ntheta, int nr, double r_body, double r_outer, double ratio) {
  if (ntheta < 2 || nr < 1 || r_outer <= r_body || ratio <= 0.0) return "bad half-cylinder parameters";
  m = Mesh();
  std::vector<double> r(nr + 1);
  double denom = (ratio == 1.0) ? nr : (std::pow(ratio, nr) - 1.0);
  for (int j = 0; j <= nr; j++) {
    double s = (ratio == 1.0) ? j / denom : (std::pow(ratio, j) - 1.0) / denom;
    r[j] = r_body + (r_outer - r_body) * s;
  }
  r[nr] = r_outer;
  const double pi = 3.14159265358979323846;
  for (int j = 0; j <= nr; j++)
    for (int i = 0; i <= ntheta; i++) {
      double th = 0.5 * pi + pi * (static_cast<double>(i) / ntheta);
      double x = r[j] * std::cos(th), y = r[j] * std::sin(th);
      if (i == 0 || i == ntheta) x = 0.0;  // cut lines exactly on x = 0
      m.points.push_back(x);
      m.points.push_back(y);
      m.points.push_back(0.0);
    }
  auto P = [ntheta](int i, int j) { return j * (ntheta + 1) + i; };
  for (int j = 0; j < nr; j++)
    for (int i = 0; i < ntheta; i++) m.cell_nodes.push_back({P(i, j), P(i + 1, j), P(i + 1, j + 1), P(i, j + 1)});
  for (int i = 0; i < ntheta; i++) {
    m.edge_kind[edge_key(P(i, 0), P(i + 1, 0))] = BK_WALL;
    m.edge_kind[edge_key(P(i, nr), P(i + 1, nr))] = BK_INLET;
  }
  for (int j = 0; j < nr; j++) {
    m.edge_kind[edge_key(P(0, j), P(0, j + 1))] = BK_EXIT;
    m.edge_kind[edge_key(P(ntheta, j), P(ntheta, j + 1))] = BK_EXIT;
  }
  return "";
}

// Compression ramp: flat lower wall up to x_corner, then a ramp at angle_deg; the lower wall
// rises, the upper boundary stays at y = height.  open_top = 0: bounding-box classification
// (left inlet, right exit, everything else wall, as the reference reader does); open_top = 1:
// left inlet, right and top outflow, lower boundary wall.
std::string generate_ramp(Mesh &m, int nx, int ny, double length, double height, double x_corner, double angle_deg,
                          int open_top) {
  if (nx < 1 || ny < 1) return "bad ramp parameters";
  m = Mesh();
  const double t = std::tan(angle_deg * 3.14159265358979323846 / 180.0);
  for (int j = 0; j <= ny; j++)
    for (int i = 0; i <= nx; i++) {
      double x = length * (static_cast<double>(i) / nx);
      double yb = x > x_corner ? (x - x_corner) * t : 0.0;
      double y = yb + (height - yb) * (static_cast<double>(j) / ny);
      m.points.push_back(x);
      m.points.push_back(y);
      m.points.push_back(0.0);
    }
  auto P = [nx](int i, int j) { return j * (nx + 1) + i; };
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) m.cell_nodes.push_back({P(i, j), P(i + 1, j), P(i + 1, j + 1), P(i, j + 1)});
  if (open_top) {
    for (int i = 0; i < nx; i++) {
      m.edge_kind[edge_key(P(i, 0), P(i + 1, 0))] = BK_WALL;
      m.edge_kind[edge_key(P(i, ny), P(i + 1, ny))] = BK_EXIT;
    }
    for (int j = 0; j < ny; j++) {
      m.edge_kind[edge_key(P(0, j), P(0, j + 1))] = BK_INLET;
      m.edge_kind[edge_key(P(nx, j), P(nx, j + 1))] = BK_EXIT;
    }
  }
  return "";
}

namespace {
// splitmix64: small seeded generator for mesh jitter.
struct SplitMix {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
};
}  // namespace

// Channel [0, length] x [0, height] with a circular-arc bump of chord 1 centred at length/2 on
// the lower wall (thickness = max height / chord).  n_quad_layers quad rows hug each wall; the
// core rows are split into triangles (alternating diagonals) when `triangles` is set, and the
// interior core nodes are moved by a seeded displacement uniform in the disc of radius
// jitter * min(hx, hy) (rejection sampling, no transcendental functions, so the mesh is the same
// on every host).  With jitter < 0.35 no triangle of a split square can invert: its smallest
// height, h/sqrt(2), loses at most 2 * jitter * h.  Left = subsonic inflow, right = outflow,
// walls elsewhere.
std::string generate_bump(Mesh &m, int nx, int ny, double length, double height, double thickness, int n_quad_layers,
                          double jitter, uint64_t seed, int triangles) {
  if (nx < 2 || ny < 2 || thickness < 0.0) return "bad bump parameters";
  m = Mesh();
  const double xc = 0.5 * length, chord = 1.0;
  // Circular arc through (xc-0.5, 0), (xc+0.5, 0) and (xc, thickness*chord).
  const double hgt = thickness * chord;
  const double R = hgt > 0.0 ? (0.25 * chord * chord + hgt * hgt) / (2.0 * hgt) : 0.0;
  auto ybot = [&](double x) {
    if (hgt <= 0.0 || x <= xc - 0.5 * chord || x >= xc + 0.5 * chord) return 0.0;
    double dx = x - xc;
    return std::sqrt(R * R - dx * dx) - (R - hgt);
  };
  SplitMix rng{seed};
  const int nql = std::max(0, std::min(n_quad_layers, ny / 2 - 1));
  for (int j = 0; j <= ny; j++)
    for (int i = 0; i <= nx; i++) {
      double x = length * (static_cast<double>(i) / nx);
      double yb = ybot(x);
      // Cluster rows towards both walls (tanh-free quadratic blend).
      double s = static_cast<double>(j) / ny;
      double y = yb + (height - yb) * s;
      if (jitter > 0.0 && i > 0 && i < nx && j > nql && j < ny - nql) {
        const double hx = length / nx, hy = (height - yb) / ny, h = hx < hy ? hx : hy;
        double a, b;
        do {
          a = 2.0 * rng.uniform() - 1.0;
          b = 2.0 * rng.uniform() - 1.0;
        } while (a * a + b * b > 1.0);
        x += jitter * h * a;
        y += jitter * h * b;
      }
      m.points.push_back(x);
      m.points.push_back(y);
      m.points.push_back(0.0);
    }
  auto P = [nx](int i, int j) { return j * (nx + 1) + i; };
  for (int j = 0; j < ny; j++)
    for (int i = 0; i < nx; i++) {
      bool quad = !triangles || j < nql || j >= ny - nql;
      if (quad) {
        m.cell_nodes.push_back({P(i, j), P(i + 1, j), P(i + 1, j + 1), P(i, j + 1)});
      } else if ((i + j) % 2 == 0) {
        m.cell_nodes.push_back({P(i, j), P(i + 1, j), P(i + 1, j + 1)});
        m.cell_nodes.push_back({P(i, j), P(i + 1, j + 1), P(i, j + 1)});
      } else {
        m.cell_nodes.push_back({P(i, j), P(i + 1, j), P(i, j + 1)});
        m.cell_nodes.push_back({P(i + 1, j), P(i + 1, j + 1), P(i, j + 1)});
      }
    }
  for (int i = 0; i < nx; i++) {
    m.edge_kind[edge_key(P(i, 0), P(i + 1, 0))] = BK_WALL;
    m.edge_kind[edge_key(P(i, ny), P(i + 1, ny))] = BK_WALL;
  }
  for (int j = 0; j < ny; j++) {
    m.edge_kind[edge_key(P(0, j), P(0, j + 1))] = BK_INLET;
    m.edge_kind[edge_key(P(nx, j), P(nx, j + 1))] = BK_EXIT;
  }
  return "";
}

// ---------------------------------------------------------------------------------------------
// Legacy VTK I/O (ASCII UNSTRUCTURED_GRID; 2-node line cells are skipped like the reference does)
// ---------------------------------------------------------------------------------------------

std::string read_vtk(Mesh &m, const std::string &path) {
  std::ifstream in(path);
  if (!in) return "cannot open " + path;
  m = Mesh();
  std::string line;
  int ncells = 0;
  while (std::getline(in, line)) {
    std::stringstream ss(line);
    std::string kw;
    ss >> kw;
    if (kw == "POINTS") {
      int n = 0;
      ss >> n;
      m.points.resize(static_cast<size_t>(n) * 3);
      for (int i = 0; i < 3 * n; i++) {
        std::string tok;
        in >> tok;
        m.points[i] = std::strtod(tok.c_str(), nullptr);
      }
    } else if (kw == "CELLS") {
      ss >> ncells;
      for (int i = 0; i < ncells; i++) {
        int nn = 0;
        in >> nn;
        std::vector<int> nodes(nn);
        for (int &x : nodes) in >> x;
        if (nn == 3 || nn == 4) m.cell_nodes.push_back(nodes);
      }
    }
  }
  if (m.points.empty() || m.cell_nodes.empty()) return "no POINTS/CELLS in " + path;
  return "";
}

std::string write_vtk(const Mesh &m, const std::string &path) {
  FILE *f = std::fopen(path.c_str(), "w");
  if (!f) return "cannot write " + path;
  size_t np = m.points.size() / 3;
  std::fprintf(f, "# vtk DataFile Version 2.0\ncfd-b200 mesh\nASCII\nDATASET UNSTRUCTURED_GRID\n");
  std::fprintf(f, "POINTS %zu double\n", np);
  for (size_t i = 0; i < np; i++)
    std::fprintf(f, "%.17g %.17g %.17g\n", m.points[3 * i], m.points[3 * i + 1], m.points[3 * i + 2]);
  size_t total = 0;
  for (const auto &c : m.cell_nodes) total += c.size() + 1;
  std::fprintf(f, "CELLS %zu %zu\n", m.cell_nodes.size(), total);
  for (const auto &c : m.cell_nodes) {
    std::fprintf(f, "%zu", c.size());
    for (int n : c) std::fprintf(f, " %d", n);
    std::fprintf(f, "\n");
  }
  std::fprintf(f, "CELL_TYPES %zu\n", m.cell_nodes.size());
  for (const auto &c : m.cell_nodes) std::fprintf(f, "%d\n", c.size() == 4 ? 9 : 5);
  std::fclose(f);
  return "";
}

// ---------------------------------------------------------------------------------------------
// Reverse Cuthill-McKee over the physical-cell adjacency (ghosts excluded).
// ---------------------------------------------------------------------------------------------

}  // namespace cfdb
