// ORACLE — test infrastructure only. This is a CPU restatement of larsbrubaker/solidfem's solve
// path (mesh -> Tet10 -> load -> stiffness -> block smoothed-aggregation multigrid -> PCG ->
// stress recovery), written to reproduce the reference's floating-point results to the bit. It is
// the checker for the CUDA product in solidfem_b200/ and the timed CPU baseline; the product never
// links, imports or calls it. Compile with -ffp-contract=off (the reference never fuses a multiply
// and an add) on x86-64 SSE2.
//
// Parity is pinned by the reference's own golden fingerprints
// (crates/solidfem/tests/validation/multigrid_precision.rs:231-250), checked by
// tests/test_oracle_pins.py.
//
// Every function cites the reference file:line it restates (paths inside the reference project).

#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle.h"

namespace orc {

using std::array;
using std::size_t;
using std::vector;
typedef array<double, 3> P3;

static const uint32_t FIXED = 0xffffffffu;       // crates/solidfem-elastic/src/assembly.rs:15
static const uint32_t NO_AGGREGATE = 0xffffffffu; // crates/solidfem-solve/src/multigrid/aggregate.rs:14
static const size_t MIN_PARALLEL_VALUES = 100000; // crates/solidfem-solve/src/parallel.rs:29

// ---------------------------------------------------------------------------------------------
// Mesh: crates/solidfem-mesh/src/{box_mesh,tet,quadratic,boundary}.rs
// ---------------------------------------------------------------------------------------------

// boundary.rs:8-13
static const int FACE_NODES[4][6] = {
    {1, 2, 3, 5, 9, 8}, {0, 3, 2, 7, 9, 6}, {0, 1, 3, 4, 8, 7}, {0, 2, 1, 6, 5, 4}};
// quadratic.rs:10 / shape.rs:23
static const int EDGE_CORNERS[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};

struct TetMesh {
  vector<P3> positions;
  vector<array<uint32_t, 4>> tets;
};

// tet.rs:9-16
static double tet_volume(const P3& a, const P3& b, const P3& c, const P3& d) {
  double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  double v[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  double w[3] = {d[0] - a[0], d[1] - a[1], d[2] - a[2]};
  double det = u[0] * (v[1] * w[2] - v[2] * w[1]) - u[1] * (v[0] * w[2] - v[2] * w[0]) +
               u[2] * (v[0] * w[1] - v[1] * w[0]);
  return det / 6.0;
}

// tet.rs:28-44
static double relative_volume(const P3& a, const P3& b, const P3& c, const P3& d, double volume) {
  auto ls = [](const P3& p, const P3& q) {
    return (p[0] - q[0]) * (p[0] - q[0]) + (p[1] - q[1]) * (p[1] - q[1]) +
           (p[2] - q[2]) * (p[2] - q[2]);
  };
  double l[6] = {ls(a, b), ls(a, c), ls(a, d), ls(b, c), ls(b, d), ls(c, d)};
  double longest = 0.0;
  for (double x : l) longest = std::max(longest, x);
  return 6.0 * volume / (longest * std::sqrt(longest));
}

static array<uint32_t, 3> sorted_key(array<uint32_t, 3> c) {
  std::sort(c.begin(), c.end());
  return c;
}

static array<uint32_t, 3> face_corners(const array<uint32_t, 4>& tet, int face) {
  return {tet[FACE_NODES[face][0]], tet[FACE_NODES[face][1]], tet[FACE_NODES[face][2]]};
}

// tet.rs:59-109. Returns 0 or an ORC_MESH_* code.
static int validate_mesh(const TetMesh& m) {
  if (m.tets.empty()) return ORC_MESH_EMPTY;
  for (auto& p : m.positions)
    for (double c : p)
      if (!std::isfinite(c)) return ORC_MESH_NONFINITE;
  vector<char> used(m.positions.size(), 0);
  for (auto& t : m.tets) {
    for (uint32_t n : t) {
      if (n >= m.positions.size()) return ORC_MESH_NODE_RANGE;
      used[n] = 1;
    }
    const P3 &a = m.positions[t[0]], &b = m.positions[t[1]], &c = m.positions[t[2]],
             &d = m.positions[t[3]];
    double volume = tet_volume(a, b, c, d);
    if (std::isnan(volume) || volume <= 0.0) return ORC_MESH_DEGENERATE;
    double rel = relative_volume(a, b, c, d, volume);
    if (std::isnan(rel) || rel < 1e-12) return ORC_MESH_FLAT;
  }
  for (char u : used)
    if (!u) return ORC_MESH_UNUSED;
  vector<array<uint32_t, 3>> faces;
  faces.reserve(m.tets.size() * 4);
  for (auto& t : m.tets)
    for (int f = 0; f < 4; ++f) faces.push_back(sorted_key(face_corners(t, f)));
  std::sort(faces.begin(), faces.end());
  for (size_t i = 0; i + 2 < faces.size(); ++i)
    if (faces[i] == faces[i + 2]) return ORC_MESH_NONMANIFOLD;
  return 0;
}

// box_mesh.rs:84-90
static double coord(double origin, double size, size_t index, size_t divisions) {
  if (index == divisions) return origin + size;
  return origin + size * ((double)index / (double)divisions);
}

// box_mesh.rs:22-80
static int box_tet_mesh(const double origin[3], const double size[3], const size_t div[3],
                        TetMesh& out) {
  for (int a = 0; a < 3; ++a)
    if (div[a] == 0) return ORC_MESH_BOX;
  for (int a = 0; a < 3; ++a)
    if (std::isnan(size[a]) || size[a] <= 0.0) return ORC_MESH_BOX;
  size_t dims[3] = {div[0] + 1, div[1] + 1, div[2] + 1};
  auto node_index = [&](size_t i, size_t j, size_t k) {
    return (uint32_t)(i + dims[0] * (j + dims[1] * k));
  };
  out.positions.clear();
  out.positions.reserve(dims[0] * dims[1] * dims[2]);
  for (size_t k = 0; k < dims[2]; ++k)
    for (size_t j = 0; j < dims[1]; ++j)
      for (size_t i = 0; i < dims[0]; ++i)
        out.positions.push_back({coord(origin[0], size[0], i, div[0]),
                                 coord(origin[1], size[1], j, div[1]),
                                 coord(origin[2], size[2], k, div[2])});
  static const int ORDERS[6][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1},
                                   {0, 2, 1}, {2, 1, 0}, {1, 0, 2}};
  static const bool EVEN[6] = {true, true, true, false, false, false};
  out.tets.clear();
  out.tets.reserve(6 * div[0] * div[1] * div[2]);
  for (size_t k = 0; k < div[2]; ++k)
    for (size_t j = 0; j < div[1]; ++j)
      for (size_t i = 0; i < div[0]; ++i)
        for (int o = 0; o < 6; ++o) {
          size_t at[3] = {i, j, k};
          uint32_t v0 = node_index(at[0], at[1], at[2]);
          at[ORDERS[o][0]] += 1;
          uint32_t v1 = node_index(at[0], at[1], at[2]);
          at[ORDERS[o][1]] += 1;
          uint32_t v2 = node_index(at[0], at[1], at[2]);
          at[ORDERS[o][2]] += 1;
          uint32_t v3 = node_index(at[0], at[1], at[2]);
          if (EVEN[o])
            out.tets.push_back({v0, v1, v2, v3});
          else
            out.tets.push_back({v0, v2, v1, v3});
        }
  return validate_mesh(out);
}

struct QuadMesh {
  vector<P3> nodes;
  vector<array<uint32_t, 10>> tets;
  vector<array<uint32_t, 4>> corner_tets;
  size_t vertex_count = 0;
};

// quadratic.rs:24-71
static QuadMesh from_linear(const TetMesh& mesh) {
  QuadMesh q;
  q.vertex_count = mesh.positions.size();
  vector<uint64_t> edges;
  edges.reserve(mesh.tets.size() * 6);
  for (auto& t : mesh.tets)
    for (int e = 0; e < 6; ++e) {
      uint32_t x = t[EDGE_CORNERS[e][0]], y = t[EDGE_CORNERS[e][1]];
      edges.push_back(((uint64_t)std::min(x, y) << 32) | std::max(x, y));
    }
  std::sort(edges.begin(), edges.end());
  edges.erase(std::unique(edges.begin(), edges.end()), edges.end());
  q.nodes = mesh.positions;
  q.nodes.reserve(q.nodes.size() + edges.size());
  for (uint64_t e : edges) {
    P3 p = q.nodes[e >> 32], r = q.nodes[e & 0xffffffffu];
    q.nodes.push_back({0.5 * (p[0] + r[0]), 0.5 * (p[1] + r[1]), 0.5 * (p[2] + r[2])});
  }
  q.tets.reserve(mesh.tets.size());
  for (auto& t : mesh.tets) {
    array<uint32_t, 10> quad;
    for (int i = 0; i < 4; ++i) quad[i] = t[i];
    for (int e = 0; e < 6; ++e) {
      uint32_t x = t[EDGE_CORNERS[e][0]], y = t[EDGE_CORNERS[e][1]];
      uint64_t key = ((uint64_t)std::min(x, y) << 32) | std::max(x, y);
      size_t at = std::lower_bound(edges.begin(), edges.end(), key) - edges.begin();
      quad[4 + e] = (uint32_t)(q.vertex_count + at);
    }
    q.tets.push_back(quad);
  }
  q.corner_tets = mesh.tets;
  return q;
}

struct BoundaryFace {
  uint32_t tet;
  uint8_t face;
  array<uint32_t, 6> nodes;
};

// quadratic.rs:89-124
static vector<BoundaryFace> boundary_faces(const QuadMesh& q) {
  struct Key {
    array<uint32_t, 3> key;
    size_t tet;
    size_t face;
    bool operator<(const Key& o) const {
      if (key != o.key) return key < o.key;
      if (tet != o.tet) return tet < o.tet;
      return face < o.face;
    }
  };
  vector<Key> keyed;
  keyed.reserve(q.tets.size() * 4);
  for (size_t t = 0; t < q.corner_tets.size(); ++t)
    for (size_t f = 0; f < 4; ++f)
      keyed.push_back({sorted_key(face_corners(q.corner_tets[t], (int)f)), t, f});
  std::sort(keyed.begin(), keyed.end());
  vector<BoundaryFace> boundary;
  size_t at = 0;
  while (at < keyed.size()) {
    size_t end = at + 1;
    while (end < keyed.size() && keyed[end].key == keyed[at].key) ++end;
    if (end == at + 1) {
      BoundaryFace bf;
      bf.tet = (uint32_t)keyed[at].tet;
      bf.face = (uint8_t)keyed[at].face;
      for (int s = 0; s < 6; ++s) bf.nodes[s] = q.tets[keyed[at].tet][FACE_NODES[keyed[at].face][s]];
      boundary.push_back(bf);
    }
    at = end;
  }
  return boundary;
}

// quadratic.rs:129-166
static vector<vector<uint32_t>> face_connected_bodies(const QuadMesh& q) {
  vector<size_t> parent(q.tets.size());
  for (size_t i = 0; i < parent.size(); ++i) parent[i] = i;
  auto find = [&](size_t x) {
    while (parent[x] != x) {
      parent[x] = parent[parent[x]];
      x = parent[x];
    }
    return x;
  };
  vector<std::pair<array<uint32_t, 3>, size_t>> keyed;
  for (size_t t = 0; t < q.corner_tets.size(); ++t)
    for (int f = 0; f < 4; ++f) keyed.push_back({sorted_key(face_corners(q.corner_tets[t], f)), t});
  std::sort(keyed.begin(), keyed.end());
  for (size_t i = 0; i + 1 < keyed.size(); ++i)
    if (keyed[i].first == keyed[i + 1].first) {
      size_t a = find(keyed[i].second), b = find(keyed[i + 1].second);
      if (a != b) {
        if (a < b)
          parent[b] = a;
        else
          parent[a] = b;
      }
    }
  vector<vector<uint32_t>> groups;
  vector<size_t> group_of_root(q.tets.size(), SIZE_MAX);
  for (size_t t = 0; t < q.tets.size(); ++t) {
    size_t root = find(t);
    if (group_of_root[root] == SIZE_MAX) {
      group_of_root[root] = groups.size();
      groups.emplace_back();
    }
    groups[group_of_root[root]].push_back((uint32_t)t);
  }
  return groups;
}

// ---------------------------------------------------------------------------------------------
// Element: crates/solidfem-elastic/src/{shape,quadrature,material,element}.rs
// ---------------------------------------------------------------------------------------------

struct QPoint {
  double natural[3];
  double weight;
};

// quadrature.rs:111-118
static const double A4 = 0.1381966011250105;
static const double B4 = 0.5854101966249685;
static const QPoint FOUR_POINT[4] = {
    {{A4, A4, A4}, 0.25}, {{B4, A4, A4}, 0.25}, {{A4, B4, A4}, 0.25}, {{A4, A4, B4}, 0.25}};
// quadrature.rs:120-144
static const double A14 = 0.3108859192633006;
static const double B14 = 1.0 - 3.0 * A14;
static const double W14A = 0.11268792571801585;
static const double C14 = 0.09273525031089123;
static const double D14 = 1.0 - 3.0 * C14;
static const double W14B = 0.07349304311636195;
static const double E14 = 0.04550370412564965;
static const double F14 = 0.5 - E14;
static const double W14C = 0.042546020777081466;
static const QPoint FOURTEEN_POINT[14] = {
    {{A14, A14, A14}, W14A}, {{B14, A14, A14}, W14A}, {{A14, B14, A14}, W14A},
    {{A14, A14, B14}, W14A}, {{C14, C14, C14}, W14B}, {{D14, C14, C14}, W14B},
    {{C14, D14, C14}, W14B}, {{C14, C14, D14}, W14B}, {{E14, E14, F14}, W14C},
    {{E14, F14, E14}, W14C}, {{F14, E14, E14}, W14C}, {{E14, F14, F14}, W14C},
    {{F14, E14, F14}, W14C}, {{F14, F14, E14}, W14C}};
// quadrature.rs:146-161
static const double TA = 0.091576213509771;
static const double TB = 0.445948490915965;
static const double WA = 0.109951743655322;
static const double WB = 0.223381589678011;
static const double TRIANGLE[6][3] = {{TA, TA, WA},
                                      {1.0 - 2.0 * TA, TA, WA},
                                      {TA, 1.0 - 2.0 * TA, WA},
                                      {TB, TB, WB},
                                      {1.0 - 2.0 * TB, TB, WB},
                                      {TB, 1.0 - 2.0 * TB, WB}};

// shape.rs:9-20
static const double NODE_NATURAL[10][3] = {{0, 0, 0},     {1, 0, 0},     {0, 1, 0},   {0, 0, 1},
                                           {0.5, 0, 0},   {0.5, 0.5, 0}, {0, 0.5, 0}, {0, 0, 0.5},
                                           {0.5, 0, 0.5}, {0, 0.5, 0.5}};

static void rule_points(int quadrature, const QPoint** pts, int* count) {
  if (quadrature == 1) {
    *pts = FOURTEEN_POINT;
    *count = 14;
  } else {
    *pts = FOUR_POINT;
    *count = 4;
  }
}

// shape.rs:25-32
static void barycentrics(const double n[3], double l[4]) {
  l[0] = 1.0 - n[0] - n[1] - n[2];
  l[1] = n[0];
  l[2] = n[1];
  l[3] = n[2];
}

// shape.rs:35-45
static void shape_values(const double nat[3], double n[10]) {
  double l[4];
  barycentrics(nat, l);
  for (int i = 0; i < 4; ++i) n[i] = l[i] * (2.0 * l[i] - 1.0);
  for (int e = 0; e < 6; ++e) n[4 + e] = 4.0 * l[EDGE_CORNERS[e][0]] * l[EDGE_CORNERS[e][1]];
}

// shape.rs:48-67
static void shape_derivatives(const double nat[3], double d[10][3]) {
  double l[4];
  barycentrics(nat, l);
  static const double DL[4][3] = {{-1.0, -1.0, -1.0}, {1.0, 0.0, 0.0}, {0.0, 1.0, 0.0},
                                  {0.0, 0.0, 1.0}};
  for (int axis = 0; axis < 3; ++axis) {
    for (int i = 0; i < 4; ++i) d[i][axis] = (4.0 * l[i] - 1.0) * DL[i][axis];
    for (int e = 0; e < 6; ++e) {
      int a = EDGE_CORNERS[e][0], b = EDGE_CORNERS[e][1];
      d[4 + e][axis] = 4.0 * (DL[a][axis] * l[b] + l[a] * DL[b][axis]);
    }
  }
}

struct Geometry {
  double gradients[10][3];
  double det_j;
  double position[3];
};

// element.rs:25-80. Returns false for an inverted point.
static bool point_geometry(const P3 nodes[10], const double nat[3], Geometry& g) {
  double der[10][3], val[10];
  shape_derivatives(nat, der);
  shape_values(nat, val);
  double j[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  double pos[3] = {0, 0, 0};
  for (int a = 0; a < 10; ++a)
    for (int i = 0; i < 3; ++i) {
      for (int k = 0; k < 3; ++k) j[i][k] += der[a][i] * nodes[a][k];
      pos[i] += val[a] * nodes[a][i];
    }
  double cof[3][3] = {{j[1][1] * j[2][2] - j[1][2] * j[2][1], j[0][2] * j[2][1] - j[0][1] * j[2][2],
                       j[0][1] * j[1][2] - j[0][2] * j[1][1]},
                      {j[1][2] * j[2][0] - j[1][0] * j[2][2], j[0][0] * j[2][2] - j[0][2] * j[2][0],
                       j[0][2] * j[1][0] - j[0][0] * j[1][2]},
                      {j[1][0] * j[2][1] - j[1][1] * j[2][0], j[0][1] * j[2][0] - j[0][0] * j[2][1],
                       j[0][0] * j[1][1] - j[0][1] * j[1][0]}};
  double det = j[0][0] * cof[0][0] + j[0][1] * cof[1][0] + j[0][2] * cof[2][0];
  g.det_j = det;
  for (int i = 0; i < 3; ++i) g.position[i] = pos[i];
  if (std::isnan(det) || det <= 0.0) return false;
  for (int a = 0; a < 10; ++a)
    for (int k = 0; k < 3; ++k) {
      double sum = cof[k][0] * der[a][0] + cof[k][1] * der[a][1] + cof[k][2] * der[a][2];
      g.gradients[a][k] = sum / det;
    }
  return true;
}

struct Material {
  double E, nu;
  bool valid() const { return std::isfinite(E) && E > 0.0 && nu > -1.0 && nu < 0.5; }
  // material.rs:24-31
  void lame(double& lambda, double& mu) const {
    lambda = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    mu = E / (2.0 * (1.0 + nu));
  }
};

// The material fields the oracle can express; the reference takes any `MaterialField`
// (material.rs:35-50) and evaluates it at each integration point by position.
struct MaterialField {
  orc_material spec;
  Material at(const double p[3]) const {
    if (spec.kind == ORC_MATERIAL_SHELL_CORE) {
      double depth = INFINITY;
      for (int a = 0; a < 3; ++a) {
        depth = std::min(depth, p[a] - spec.lo[a]);
        depth = std::min(depth, spec.hi[a] - p[a]);
      }
      if (depth < spec.depth) return {spec.E, spec.nu};
      return {spec.E2, spec.nu2};
    }
    return {spec.E, spec.nu};
  }
};

// element.rs:98-133. Returns 0, or ORC_ELEMENT_INVERTED / ORC_ELEMENT_MATERIAL.
static int element_stiffness(const P3 nodes[10], const MaterialField& field, int quadrature,
                             double ke[900]) {
  std::fill(ke, ke + 900, 0.0);
  const QPoint* pts;
  int count;
  rule_points(quadrature, &pts, &count);
  for (int qi = 0; qi < count; ++qi) {
    Geometry g;
    if (!point_geometry(nodes, pts[qi].natural, g)) return ORC_ELEMENT_INVERTED;
    Material m = field.at(g.position);
    if (!m.valid()) return ORC_ELEMENT_MATERIAL;
    double lambda, mu;
    m.lame(lambda, mu);
    double measure = pts[qi].weight * g.det_j / 6.0;
    for (int a = 0; a < 10; ++a)
      for (int b = a; b < 10; ++b) {
        const double* ga = g.gradients[a];
        const double* gb = g.gradients[b];
        double dot = ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2];
        for (int i = 0; i < 3; ++i)
          for (int k = 0; k < 3; ++k) {
            double value = lambda * (ga[i] * gb[k]) + mu * (ga[k] * gb[i]);
            if (i == k) value += mu * dot;
            value *= measure;
            ke[(3 * a + i) * 30 + (3 * b + k)] += value;
            if (a != b) ke[(3 * b + k) * 30 + (3 * a + i)] += value;
          }
      }
  }
  return 0;
}

// element.rs:159-189
static void strain_at(const Geometry& g, const double u[10][3], double strain[6]) {
  double h[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int a = 0; a < 10; ++a)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) h[i][j] += u[a][i] * g.gradients[a][j];
  strain[0] = h[0][0];
  strain[1] = h[1][1];
  strain[2] = h[2][2];
  strain[3] = h[0][1] + h[1][0];
  strain[4] = h[1][2] + h[2][1];
  strain[5] = h[2][0] + h[0][2];
}

static void stress_at(const Material& m, const double e[6], double s[6]) {
  double lambda, mu;
  m.lame(lambda, mu);
  double trace = e[0] + e[1] + e[2];
  s[0] = lambda * trace + 2.0 * mu * e[0];
  s[1] = lambda * trace + 2.0 * mu * e[1];
  s[2] = lambda * trace + 2.0 * mu * e[2];
  s[3] = mu * e[3];
  s[4] = mu * e[4];
  s[5] = mu * e[5];
}

static double von_mises(const double s[6]) {
  double a = s[0] - s[1], b = s[1] - s[2], c = s[2] - s[0];
  return std::sqrt(0.5 * (a * a + b * b + c * c) + 3.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]));
}

// ---------------------------------------------------------------------------------------------
// Scalar CSR: crates/solidfem-solve/src/csr.rs
// ---------------------------------------------------------------------------------------------

struct Csr {
  size_t size = 0;
  vector<size_t> row_starts;
  vector<uint32_t> columns;
  vector<double> values;

  // csr.rs:19-71
  static Csr from_block_connectivity(size_t block_count, size_t block_size,
                                     const vector<vector<uint32_t>>& elements) {
    vector<uint64_t> pairs;
    for (auto& el : elements)
      for (uint32_t r : el)
        for (uint32_t c : el) pairs.push_back(((uint64_t)r << 32) | c);
    std::sort(pairs.begin(), pairs.end());
    pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
    Csr m;
    m.size = block_count * block_size;
    vector<size_t> block_rows(block_count + 1, 0);
    for (uint64_t p : pairs) block_rows[(p >> 32) + 1] += 1;
    for (size_t i = 0; i < block_count; ++i) block_rows[i + 1] += block_rows[i];
    m.row_starts.reserve(m.size + 1);
    m.columns.reserve(pairs.size() * block_size * block_size);
    m.row_starts.push_back(0);
    for (size_t b = 0; b < block_count; ++b)
      for (size_t r = 0; r < block_size; ++r) {
        for (size_t at = block_rows[b]; at < block_rows[b + 1]; ++at) {
          size_t cb = (size_t)(pairs[at] & 0xffffffffu);
          for (size_t o = 0; o < block_size; ++o) m.columns.push_back((uint32_t)(cb * block_size + o));
        }
        m.row_starts.push_back(m.columns.size());
      }
    m.values.assign(m.columns.size(), 0.0);
    return m;
  }

  size_t find(size_t row, uint32_t column) const {
    auto b = columns.begin() + row_starts[row], e = columns.begin() + row_starts[row + 1];
    auto it = std::lower_bound(b, e, column);
    if (it == e || *it != column) return SIZE_MAX;
    return (size_t)(it - columns.begin());
  }
  // csr.rs:89-96
  void add(size_t row, uint32_t column, double v) { values[find(row, column)] += v; }
  // csr.rs:99-105
  double get(size_t row, uint32_t column) const {
    size_t at = find(row, column);
    return at == SIZE_MAX ? 0.0 : values[at];
  }
  // csr.rs:124-132
  void multiply_rows(size_t r0, size_t r1, const double* x, double* y) const {
    for (size_t row = r0; row < r1; ++row) {
      double sum = 0.0;
      for (size_t at = row_starts[row]; at < row_starts[row + 1]; ++at)
        sum += values[at] * x[columns[at]];
      y[row - r0] = sum;
    }
  }
  // csr.rs:142-154
  double multiply_rounding_bound(const double* x) const {
    double sum = 0.0;
    for (size_t row = 0; row < size; ++row) {
      size_t s = row_starts[row], e = row_starts[row + 1];
      double row_sum = 0.0;
      for (size_t at = s; at < e; ++at) row_sum += std::fabs(values[at] * x[columns[at]]);
      double bound = (double)(e - s) * 2.220446049250313e-16 * row_sum;
      sum += bound * bound;
    }
    return std::sqrt(sum);
  }
};

// Row-parallel helper: every row is a pure function of its own data, so any partition gives the
// bits of a serial run (crates/solidfem-solve/src/parallel.rs:5-10).
static int g_threads = 1;
template <class F>
static void for_rows(size_t rows, bool parallel, F&& f) {
#ifdef _OPENMP
  if (parallel && g_threads > 1) {
#pragma omp parallel for schedule(static) num_threads(g_threads)
    for (long long r = 0; r < (long long)rows; ++r) f((size_t)r);
    return;
  }
#endif
  (void)parallel;
  for (size_t r = 0; r < rows; ++r) f(r);
}

// ---------------------------------------------------------------------------------------------
// Block storage and small dense kernels: crates/solidfem-solve/src/multigrid/block.rs
// ---------------------------------------------------------------------------------------------

template <class T>
struct BlockCsr {
  size_t rows = 0, row_block = 0, col_block = 0;
  vector<size_t> starts;
  vector<uint32_t> columns;
  vector<T> values;
  size_t block_len() const { return row_block * col_block; }
  size_t dofs() const { return rows * row_block; }
  const T* block(size_t at) const { return values.data() + at * block_len(); }
  size_t memory_bytes() const {
    return starts.size() * sizeof(size_t) + columns.size() * sizeof(uint32_t) + values.size() * sizeof(T);
  }
  // block.rs:136-154
  template <class V>
  void multiply_row(size_t row, const V* x, V* out) const {
    size_t rb = row_block, cb = col_block;
    for (size_t p = 0; p < rb; ++p) out[p] = V(0);
    for (size_t at = starts[row]; at < starts[row + 1]; ++at) {
      const T* b = block(at);
      size_t col = (size_t)columns[at] * cb;
      for (size_t p = 0; p < rb; ++p) {
        V sum = out[p];
        for (size_t q = 0; q < cb; ++q) sum += (V)b[p * cb + q] * x[col + q];
        out[p] = sum;
      }
    }
  }
  template <class V>
  void multiply(const V* x, V* y, bool parallel = false) const {
    for_rows(rows, parallel, [&](size_t r) { multiply_row(r, x, y + r * row_block); });
  }
  // block.rs:157-172
  template <class V>
  void multiply_transpose(const V* x, V* y, size_t out_len) const {
    size_t rb = row_block, cb = col_block;
    for (size_t i = 0; i < out_len; ++i) y[i] = V(0);
    for (size_t row = 0; row < rows; ++row)
      for (size_t at = starts[row]; at < starts[row + 1]; ++at) {
        const T* b = block(at);
        size_t col = (size_t)columns[at] * cb;
        for (size_t p = 0; p < rb; ++p) {
          V value = x[row * rb + p];
          for (size_t q = 0; q < cb; ++q) y[col + q] += (V)b[p * cb + q] * value;
        }
      }
  }
};

template <class U>
static BlockCsr<U> to_precision(const BlockCsr<double>& m) {
  BlockCsr<U> o;
  o.rows = m.rows;
  o.row_block = m.row_block;
  o.col_block = m.col_block;
  o.starts = m.starts;
  o.columns = m.columns;
  o.values.resize(m.values.size());
  for (size_t i = 0; i < m.values.size(); ++i) o.values[i] = (U)m.values[i];
  return o;
}

// block.rs:51-99
static int from_nodal(const Csr& m, BlockCsr<double>& b) {
  if (m.size % 3 != 0) return ORC_MG_BLOCK_STRUCTURE;
  size_t rows = m.size / 3;
  b = BlockCsr<double>();
  b.rows = rows;
  b.row_block = 3;
  b.col_block = 3;
  b.starts.push_back(0);
  b.columns.reserve(m.columns.size() / 9);
  b.values.reserve(m.columns.size());
  for (size_t node = 0; node < rows; ++node) {
    size_t s[3], e[3];
    for (int i = 0; i < 3; ++i) {
      s[i] = m.row_starts[3 * node + i];
      e[i] = m.row_starts[3 * node + i + 1];
    }
    size_t len = e[0] - s[0];
    for (int i = 1; i < 3; ++i) {
      if (e[i] - s[i] != len) return ORC_MG_BLOCK_STRUCTURE;
      for (size_t k = 0; k < len; ++k)
        if (m.columns[s[i] + k] != m.columns[s[0] + k]) return ORC_MG_BLOCK_STRUCTURE;
    }
    if (len % 3 != 0) return ORC_MG_BLOCK_STRUCTURE;
    for (size_t at = 0; at < len; at += 3) {
      size_t c = m.columns[s[0] + at];
      if (c % 3 != 0 || m.columns[s[0] + at + 1] != c + 1 || m.columns[s[0] + at + 2] != c + 2)
        return ORC_MG_BLOCK_STRUCTURE;
      b.columns.push_back((uint32_t)(c / 3));
    }
    for (size_t at = 0; at < len / 3; ++at)
      for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) b.values.push_back(m.values[s[i] + 3 * at + k]);
    b.starts.push_back(b.columns.size());
  }
  return 0;
}

// block.rs:186-224. Returns true, or false with the failing pivot.
static bool invert_spd_block(const double* input, size_t n, double* output, double* pivot) {
  double lower[36] = {0};
  for (size_t i = 0; i < n; ++i)
    for (size_t j = 0; j <= i; ++j) {
      double sum = input[i * n + j];
      for (size_t k = 0; k < j; ++k) sum -= lower[i * n + k] * lower[j * n + k];
      if (i == j) {
        if (!std::isfinite(sum) || sum <= 0.0) {
          *pivot = sum;
          return false;
        }
        lower[i * n + j] = std::sqrt(sum);
      } else {
        lower[i * n + j] = sum / lower[j * n + j];
      }
    }
  double inverse[36] = {0};
  for (size_t c = 0; c < n; ++c)
    for (size_t i = c; i < n; ++i) {
      double sum = (i == c) ? 1.0 : 0.0;
      for (size_t k = c; k < i; ++k) sum -= lower[i * n + k] * inverse[k * n + c];
      inverse[i * n + c] = sum / lower[i * n + i];
    }
  for (size_t i = 0; i < n; ++i)
    for (size_t j = 0; j < n; ++j) {
      double sum = 0.0;
      for (size_t k = std::max(i, j); k < n; ++k) sum += inverse[k * n + i] * inverse[k * n + j];
      output[i * n + j] = sum;
    }
  return true;
}

// block.rs:229-245
static inline void add_product(double* out, const double* a, size_t a_rows, size_t middle,
                               const double* b, size_t b_cols) {
  for (size_t r = 0; r < a_rows; ++r)
    for (size_t m = 0; m < middle; ++m) {
      double scale = a[r * middle + m];
      for (size_t c = 0; c < b_cols; ++c) out[r * b_cols + c] += scale * b[m * b_cols + c];
    }
}

// block.rs:249-302
struct Accumulator {
  vector<uint32_t> slot;
  vector<uint32_t> touched;
  vector<double> data;
  size_t block_len;
  Accumulator(size_t columns, size_t bl) : slot(columns, 0xffffffffu), block_len(bl) {}
  void begin() {
    for (uint32_t c : touched) slot[c] = 0xffffffffu;
    touched.clear();
    data.clear();
  }
  double* entry(uint32_t column) {
    uint32_t at = slot[column];
    if (at == 0xffffffffu) {
      at = (uint32_t)touched.size();
      slot[column] = at;
      touched.push_back(column);
      data.resize(data.size() + block_len, 0.0);
    }
    return data.data() + (size_t)at * block_len;
  }
  template <class F>
  void drain_sorted(F&& emit) {
    std::sort(touched.begin(), touched.end());
    for (uint32_t c : touched) emit(c, data.data() + (size_t)slot[c] * block_len);
  }
};

// block.rs:307-374
struct DenseCholesky {
  size_t n = 0;
  vector<double> factor;
  size_t next = 0;
  // Returns 1 when finished, 0 when more columns remain, -1 on a bad pivot.
  int factor_column(size_t* column, double* pivot) {
    size_t j = next;
    if (j == n) return 1;
    for (size_t i = j; i < n; ++i) {
      double sum = factor[i * n + j];
      for (size_t k = 0; k < j; ++k) sum -= factor[i * n + k] * factor[j * n + k];
      if (i == j) {
        if (!std::isfinite(sum) || sum <= 0.0) {
          *column = j;
          *pivot = sum;
          return -1;
        }
        factor[j * n + j] = std::sqrt(sum);
      } else {
        factor[i * n + j] = sum / factor[j * n + j];
      }
    }
    next += 1;
    return next == n ? 1 : 0;
  }
  void solve(double* x) const {
    for (size_t i = 0; i < n; ++i) {
      double sum = x[i];
      for (size_t k = 0; k < i; ++k) sum -= factor[i * n + k] * x[k];
      x[i] = sum / factor[i * n + i];
    }
    for (size_t i = n; i-- > 0;) {
      double sum = x[i];
      for (size_t k = i + 1; k < n; ++k) sum -= factor[k * n + i] * x[k];
      x[i] = sum / factor[i * n + i];
    }
  }
};

// block.rs:379-382
static double start_value(size_t index) {
  uint64_t mixed = ((uint64_t)index + 1) * 0x9E3779B97F4A7C15ull;
  return 0.5 + (double)(mixed >> 11) / (double)(1ull << 53);
}
// block.rs:384-396
static void apply_block_diagonal(const double* inv, size_t block, const double* x, double* y, size_t len) {
  size_t rows = len / block;
  for (size_t r = 0; r < rows; ++r) {
    const double* d = inv + r * block * block;
    for (size_t p = 0; p < block; ++p) {
      double sum = 0.0;
      for (size_t q = 0; q < block; ++q) sum += d[p * block + q] * x[r * block + q];
      y[r * block + p] = sum;
    }
  }
}
// block.rs:398-411
static double norm2(const double* x, size_t n) {
  double sum = 0.0;
  for (size_t i = 0; i < n; ++i) sum += x[i] * x[i];
  return std::sqrt(sum);
}

// ---------------------------------------------------------------------------------------------
// Aggregation: crates/solidfem-solve/src/multigrid/aggregate.rs
// ---------------------------------------------------------------------------------------------

// aggregate.rs:17-23
static double block_norm(const double* b, size_t len) {
  double sum = 0.0;
  for (size_t i = 0; i < len; ++i) sum += b[i] * b[i];
  return std::sqrt(sum);
}
// aggregate.rs:26-31
static double squared_distance(const vector<P3>& p, size_t row, size_t column) {
  const P3 &h = p[row], &t = p[column];
  double dx = t[0] - h[0], dy = t[1] - h[1], dz = t[2] - h[2];
  return dx * dx + dy * dy + dz * dz;
}
// aggregate.rs:34-48
static void push_within(const BlockCsr<double>& m, const vector<P3>& pos, size_t row, double limit,
                        vector<uint32_t>& cols) {
  for (size_t at = m.starts[row]; at < m.starts[row + 1]; ++at) {
    size_t c = m.columns[at];
    if (c != row && squared_distance(pos, row, c) <= limit) cols.push_back((uint32_t)c);
  }
}
// aggregate.rs:53-69
static double strong_row(const BlockCsr<double>& m, const vector<P3>& pos, double reach, size_t row,
                         vector<uint32_t>& cols) {
  double closest = std::numeric_limits<double>::max();
  for (size_t at = m.starts[row]; at < m.starts[row + 1]; ++at) {
    size_t c = m.columns[at];
    if (c != row) closest = std::min(closest, squared_distance(pos, row, c));
  }
  push_within(m, pos, row, reach * reach * closest, cols);
  return closest;
}
// aggregate.rs:80-96
static void smoothing_row(const BlockCsr<double>& m, const vector<P3>& pos, double reach,
                          const vector<double>& closest, size_t row, vector<uint32_t>& cols) {
  double scale = closest[row];
  for (size_t at = m.starts[row]; at < m.starts[row + 1]; ++at) {
    size_t c = m.columns[at];
    if (c != row) scale = std::max(scale, closest[c]);
  }
  push_within(m, pos, row, reach * reach * scale, cols);
}

// aggregate.rs:99-178
struct Aggregation {
  vector<uint32_t> aggregate;
  vector<char> seeded;
  uint32_t count = 0;
  explicit Aggregation(size_t rows) : aggregate(rows, NO_AGGREGATE), seeded(rows, 0) {}
  void seed(size_t row, const uint32_t* nb, size_t n) {
    if (aggregate[row] != NO_AGGREGATE || n == 0) return;
    for (size_t i = 0; i < n; ++i)
      if (aggregate[nb[i]] != NO_AGGREGATE) return;
    uint32_t id = count++;
    aggregate[row] = id;
    seeded[row] = 1;
    for (size_t i = 0; i < n; ++i) {
      aggregate[nb[i]] = id;
      seeded[nb[i]] = 1;
    }
  }
  void join(size_t row, const BlockCsr<double>& m, const uint32_t* nb, size_t n) {
    if (aggregate[row] != NO_AGGREGATE) return;
    double best = 0.0;
    uint32_t chosen = NO_AGGREGATE;
    for (size_t at = m.starts[row]; at < m.starts[row + 1]; ++at) {
      uint32_t c = m.columns[at];
      if (!std::binary_search(nb, nb + n, c) || !seeded[c]) continue;
      double norm = block_norm(m.block(at), m.block_len());
      if (norm > best) {
        best = norm;
        chosen = aggregate[c];
      }
    }
    if (chosen != NO_AGGREGATE) aggregate[row] = chosen;
  }
  void sweep(size_t row, const uint32_t* nb, size_t n) {
    if (aggregate[row] != NO_AGGREGATE) return;
    uint32_t id = count++;
    aggregate[row] = id;
    for (size_t i = 0; i < n; ++i)
      if (aggregate[nb[i]] == NO_AGGREGATE) aggregate[nb[i]] = id;
  }
};

// ---------------------------------------------------------------------------------------------
// Transfer: crates/solidfem-solve/src/multigrid/transfer.rs
// ---------------------------------------------------------------------------------------------

static const size_t MODES = 6;

static double column_norm(const vector<double>& local, size_t rows, size_t column) {
  double sum = 0.0;
  for (size_t r = 0; r < rows; ++r) {
    double v = local[r * MODES + column];
    sum += v * v;
  }
  return std::sqrt(sum);
}

// transfer.rs:19-68
static void orthonormalize_aggregate(const uint32_t* members, size_t count, size_t row_block,
                                     const vector<double>& near_null, vector<double>& blocks,
                                     double coarse[36]) {
  size_t rows = count * row_block;
  vector<double> local(rows * MODES, 0.0);
  for (size_t m = 0; m < count; ++m) {
    const double* src = near_null.data() + (size_t)members[m] * row_block * MODES;
    for (size_t p = 0; p < row_block; ++p)
      for (size_t k = 0; k < MODES; ++k) local[(m * row_block + p) * MODES + k] = src[p * MODES + k];
  }
  std::fill(coarse, coarse + 36, 0.0);
  for (size_t column = 0; column < MODES; ++column) {
    double original = column_norm(local, rows, column);
    for (int pass = 0; pass < 2; ++pass)
      for (size_t prev = 0; prev < column; ++prev) {
        double projection = 0.0;
        for (size_t r = 0; r < rows; ++r) projection += local[r * MODES + prev] * local[r * MODES + column];
        coarse[prev * MODES + column] += projection;
        for (size_t r = 0; r < rows; ++r) {
          double value = local[r * MODES + prev];
          local[r * MODES + column] -= projection * value;
        }
      }
    double remainder = column_norm(local, rows, column);
    if (original == 0.0 || remainder <= 1e-10 * original) {
      for (size_t r = 0; r < rows; ++r) local[r * MODES + column] = 0.0;
      coarse[column * MODES + column] = 0.0;
    } else {
      for (size_t r = 0; r < rows; ++r) local[r * MODES + column] /= remainder;
      coarse[column * MODES + column] = remainder;
    }
  }
  blocks.insert(blocks.end(), local.begin(), local.end());
}

// transfer.rs:108-152
static void smooth_row(const BlockCsr<double>& m, const BlockCsr<double>& t, const uint32_t* nb,
                       size_t nn, const vector<double>& inv, double omega, size_t row,
                       Accumulator& acc, BlockCsr<double>& out) {
  size_t rb = m.row_block, cb = t.col_block, mid = m.col_block;
  acc.begin();
  size_t t_at = t.starts[row];
  uint32_t t_column = t.columns[t_at];
  acc.entry(t_column);
  for (size_t at = m.starts[row]; at < m.starts[row + 1]; ++at) {
    uint32_t column = m.columns[at];
    size_t source = (column == row || std::binary_search(nb, nb + nn, column)) ? column : row;
    for (size_t inner = t.starts[source]; inner < t.starts[source + 1]; ++inner) {
      double* o = acc.entry(t.columns[inner]);
      add_product(o, m.block(at), rb, mid, t.block(inner), cb);
    }
  }
  const double* dinv = inv.data() + row * rb * rb;
  vector<double> scaled(rb * cb);
  const double* t_block = t.block(t_at);
  acc.drain_sorted([&](uint32_t column, const double* block) {
    std::fill(scaled.begin(), scaled.end(), 0.0);
    add_product(scaled.data(), dinv, rb, rb, block, cb);
    out.columns.push_back(column);
    for (size_t at = 0; at < rb * cb; ++at) {
      double t_value = column == t_column ? t_block[at] : 0.0;
      out.values.push_back(t_value - omega * scaled[at]);
    }
  });
  out.starts.push_back(out.columns.size());
}

// transfer.rs:81-95 and 155-169
static void product_row(const BlockCsr<double>& m, const BlockCsr<double>& p, size_t row,
                        Accumulator& acc, BlockCsr<double>& out) {
  acc.begin();
  size_t rb = m.row_block, mid = m.col_block, cb = p.col_block;
  for (size_t at = m.starts[row]; at < m.starts[row + 1]; ++at) {
    size_t column = m.columns[at];
    for (size_t inner = p.starts[column]; inner < p.starts[column + 1]; ++inner) {
      double* o = acc.entry(p.columns[inner]);
      add_product(o, m.block(at), rb, mid, p.block(inner), cb);
    }
  }
  acc.drain_sorted([&](uint32_t column, const double* block) {
    out.columns.push_back(column);
    out.values.insert(out.values.end(), block, block + rb * cb);
  });
  out.starts.push_back(out.columns.size());
}

// transfer.rs:173-194
static void prolongator_columns(const BlockCsr<double>& p, size_t coarse_rows, vector<size_t>& starts,
                                vector<std::pair<uint32_t, size_t>>& entries) {
  starts.assign(coarse_rows + 1, 0);
  for (uint32_t c : p.columns) starts[c + 1] += 1;
  for (size_t i = 0; i < coarse_rows; ++i) starts[i + 1] += starts[i];
  vector<size_t> filled = starts;
  entries.assign(p.columns.size(), {0, 0});
  for (size_t row = 0; row < p.rows; ++row)
    for (size_t at = p.starts[row]; at < p.starts[row + 1]; ++at) {
      size_t c = p.columns[at];
      entries[filled[c]] = {(uint32_t)row, at};
      filled[c] += 1;
    }
}

// transfer.rs:204-238
static void galerkin_row(const BlockCsr<double>& p, const vector<size_t>& cstarts,
                         const vector<std::pair<uint32_t, size_t>>& entries,
                         const BlockCsr<double>& ap, size_t coarse_row, Accumulator& acc,
                         BlockCsr<double>& out) {
  size_t fine = p.row_block, coarse = p.col_block;
  acc.begin();
  vector<double> transposed(fine * coarse, 0.0);
  for (size_t e = cstarts[coarse_row]; e < cstarts[coarse_row + 1]; ++e) {
    uint32_t fine_row = entries[e].first;
    const double* block = p.block(entries[e].second);
    for (size_t a = 0; a < fine; ++a)
      for (size_t b = 0; b < coarse; ++b) transposed[b * fine + a] = block[a * coarse + b];
    for (size_t inner = ap.starts[fine_row]; inner < ap.starts[fine_row + 1]; ++inner) {
      double* o = acc.entry(ap.columns[inner]);
      add_product(o, transposed.data(), coarse, fine, ap.block(inner), coarse);
    }
  }
  acc.drain_sorted([&](uint32_t column, const double* block) {
    out.columns.push_back(column);
    out.values.insert(out.values.end(), block, block + coarse * coarse);
  });
  out.starts.push_back(out.columns.size());
}

// ---------------------------------------------------------------------------------------------
// Setup: crates/solidfem-solve/src/multigrid/{setup.rs,setup_aggregation.rs}. The reference's
// state machine is resumable; slicing never changes its bits (setup.rs:191-192), so the oracle
// runs each phase to completion in the same order.
// ---------------------------------------------------------------------------------------------

struct Level {
  BlockCsr<double> a;
  vector<double> inverse_diagonal;
  double lambda_min = 0, lambda_max = 0;
  bool has_prolongator = false;
  BlockCsr<double> prolongator;
  bool has_factor = false;
  DenseCholesky factor;
  vector<uint32_t> aggregates;
};

struct MgOptions {
  double reach = 3.0;
  size_t coarse_dofs = 1500;
  size_t max_levels = 12;
  size_t degree = 3;
  double range = 30.0;
  int precision = ORC_PRECISION_SINGLE_STORAGE;
};

struct SetupError {
  int code = 0;
  size_t level = 0, block = 0;
  double pivot = 0;
};

static bool build_hierarchy(const Csr& matrix, const vector<double>& near_null_in,
                            const vector<P3>& positions_in, const MgOptions& opt,
                            vector<Level>& levels, SetupError& err) {
  const size_t DENSE_LIMIT = 3000;            // setup.rs:28
  const double MAX_COARSE_FRACTION = 0.7;     // setup.rs:32
  const double RETRY_WIDENING = 1.5;          // setup.rs:36
  const size_t MAX_RETRIES = 3;               // setup.rs:37
  const size_t POWER_ITERATIONS = 20;         // setup.rs:41
  const double SPECTRAL_MARGIN = 1.15;        // setup.rs:45
  if (near_null_in.size() != MODES * matrix.size) {
    err.code = ORC_MG_NEAR_NULL_LENGTH;
    return false;
  }
  BlockCsr<double> current;
  if (int c = from_nodal(matrix, current)) {
    err.code = c;
    return false;
  }
  if (positions_in.size() != current.rows) {
    err.code = ORC_MG_POSITION_LENGTH;
    return false;
  }
  vector<double> near_null = near_null_in;
  vector<P3> positions = positions_in;
  levels.clear();
  while (true) {
    size_t level_index = levels.size();
    size_t rb = current.row_block;
    // Diagonal, setup.rs:269-321
    vector<double> inv(current.rows * rb * rb, 0.0);
    for (size_t row = 0; row < current.rows; ++row) {
      auto b = current.columns.begin() + current.starts[row];
      auto e = current.columns.begin() + current.starts[row + 1];
      auto it = std::lower_bound(b, e, (uint32_t)row);
      if (it == e || *it != row) {
        err = {ORC_MG_NOT_POSITIVE_DEFINITE, level_index, row, 0.0};
        return false;
      }
      size_t at = (size_t)(it - current.columns.begin());
      double pivot;
      if (!invert_spd_block(current.block(at), rb, inv.data() + row * rb * rb, &pivot)) {
        err = {ORC_MG_NOT_POSITIVE_DEFINITE, level_index, row, pivot};
        return false;
      }
    }
    bool is_coarsest =
        current.dofs() <= opt.coarse_dofs || level_index + 1 >= opt.max_levels;
    double reach = opt.reach;
    size_t retries = 0;
    vector<size_t> strong_starts;
    vector<uint32_t> strong_columns;
    vector<double> closest;
    std::unique_ptr<Aggregation> agg;
    vector<size_t> member_starts;
    vector<uint32_t> members;
    vector<P3> coarse_positions;
    if (!is_coarsest) {
      while (true) {
        // Strength, setup_aggregation.rs:12-43
        strong_starts.assign(1, 0);
        strong_columns.clear();
        closest.clear();
        for (size_t row = 0; row < current.rows; ++row) {
          closest.push_back(strong_row(current, positions, reach, row, strong_columns));
          strong_starts.push_back(strong_columns.size());
        }
        agg.reset(new Aggregation(current.rows));
        // Seed, Join, Sweep: setup_aggregation.rs:86-162
        for (size_t row = 0; row < current.rows; ++row)
          agg->seed(row, strong_columns.data() + strong_starts[row],
                    strong_starts[row + 1] - strong_starts[row]);
        for (size_t row = 0; row < current.rows; ++row)
          agg->join(row, current, strong_columns.data() + strong_starts[row],
                    strong_starts[row + 1] - strong_starts[row]);
        for (size_t row = 0; row < current.rows; ++row)
          agg->sweep(row, strong_columns.data() + strong_starts[row],
                     strong_starts[row + 1] - strong_starts[row]);
        // Group, setup_aggregation.rs:165-228
        size_t aggregates = agg->count;
        double coarse_values = (double)(aggregates * MODES);
        bool coarsens = coarse_values <= MAX_COARSE_FRACTION * (double)current.dofs();
        if (!coarsens && retries < MAX_RETRIES) {
          retries += 1;
          reach *= RETRY_WIDENING;
          continue;
        }
        if (!coarsens || aggregates == 0) {
          is_coarsest = true;
          break;
        }
        member_starts.assign(aggregates + 1, 0);
        for (uint32_t a : agg->aggregate) member_starts[a + 1] += 1;
        for (size_t i = 0; i < aggregates; ++i) member_starts[i + 1] += member_starts[i];
        vector<size_t> filled = member_starts;
        members.assign(current.rows, 0);
        for (size_t row = 0; row < current.rows; ++row) {
          uint32_t a = agg->aggregate[row];
          members[filled[a]] = (uint32_t)row;
          filled[a] += 1;
        }
        coarse_positions.assign(aggregates, {0.0, 0.0, 0.0});
        for (size_t a = 0; a < aggregates; ++a) {
          for (size_t k = member_starts[a]; k < member_starts[a + 1]; ++k) {
            const P3& p = positions[members[k]];
            for (int ax = 0; ax < 3; ++ax) coarse_positions[a][ax] += p[ax];
          }
          double count = (double)(member_starts[a + 1] - member_starts[a]);
          for (int ax = 0; ax < 3; ++ax) coarse_positions[a][ax] /= count;
        }
        break;
      }
    }
    // Tentative, setup.rs:327-386
    BlockCsr<double> tentative;
    vector<double> coarse_null;
    size_t aggregates = (!is_coarsest && agg) ? agg->count : 0;
    if (!is_coarsest) {
      size_t block = rb * MODES;
      vector<double> tvals;
      tvals.reserve(current.rows * block);
      vector<size_t> tpos(current.rows, 0);
      coarse_null.reserve(aggregates * 36);
      for (size_t a = 0; a < aggregates; ++a) {
        size_t start = tvals.size();
        double coarse[36];
        orthonormalize_aggregate(members.data() + member_starts[a], member_starts[a + 1] - member_starts[a],
                                 rb, near_null, tvals, coarse);
        for (size_t k = member_starts[a]; k < member_starts[a + 1]; ++k)
          tpos[members[k]] = start + (k - member_starts[a]) * block;
        coarse_null.insert(coarse_null.end(), coarse, coarse + 36);
      }
      tentative.rows = current.rows;
      tentative.row_block = rb;
      tentative.col_block = MODES;
      tentative.starts.push_back(0);
      for (size_t row = 0; row < current.rows; ++row) {
        tentative.columns.push_back(agg->aggregate[row]);
        tentative.values.insert(tentative.values.end(), tvals.begin() + tpos[row],
                                tvals.begin() + tpos[row] + block);
        tentative.starts.push_back(tentative.columns.size());
      }
    }
    // Spectral, setup.rs:390-449
    size_t dofs = current.dofs();
    vector<double> v(dofs), s1(dofs), s2(dofs);
    for (size_t i = 0; i < dofs; ++i) v[i] = start_value(i);
    {
      double n = norm2(v.data(), dofs);
      for (size_t i = 0; i < dofs; ++i) v[i] /= n;
    }
    double lambda_max = 0.0;
    for (size_t it = 0; it < POWER_ITERATIONS; ++it) {
      current.multiply(v.data(), s1.data());
      apply_block_diagonal(inv.data(), rb, s1.data(), s2.data(), dofs);
      double n = norm2(s2.data(), dofs);
      lambda_max = n;
      for (size_t i = 0; i < dofs; ++i) v[i] = s2[i] / n;
    }
    lambda_max *= SPECTRAL_MARGIN;
    double lambda_min = lambda_max / opt.range;
    if (is_coarsest) {
      Level lv;
      lv.a = std::move(current);
      lv.inverse_diagonal = std::move(inv);
      lv.lambda_min = lambda_min;
      lv.lambda_max = lambda_max;
      if (lv.a.dofs() <= DENSE_LIMIT) {
        // begin_factor + run_factor, setup.rs:451-504
        size_t n = lv.a.dofs();
        size_t lrb = lv.a.row_block, lcb = lv.a.col_block;
        lv.factor.n = n;
        lv.factor.factor.assign(n * n, 0.0);
        for (size_t row = 0; row < lv.a.rows; ++row)
          for (size_t at = lv.a.starts[row]; at < lv.a.starts[row + 1]; ++at) {
            size_t col = lv.a.columns[at];
            const double* b = lv.a.block(at);
            for (size_t p = 0; p < lrb; ++p)
              for (size_t q = 0; q < lcb; ++q)
                lv.factor.factor[(row * lrb + p) * n + col * lcb + q] = b[p * lcb + q];
          }
        while (true) {
          size_t column;
          double pivot;
          int r = lv.factor.factor_column(&column, &pivot);
          if (r < 0) {
            err = {ORC_MG_NOT_POSITIVE_DEFINITE, level_index, column, pivot};
            return false;
          }
          if (r == 1) break;
        }
        lv.has_factor = true;
      }
      levels.push_back(std::move(lv));
      return true;
    }
    // Filter, setup_aggregation.rs:48-84 (coarse levels only)
    vector<size_t> filter_starts;
    vector<uint32_t> filter_columns;
    if (level_index > 0) {
      filter_starts.push_back(0);
      for (size_t row = 0; row < current.rows; ++row) {
        smoothing_row(current, positions, reach, closest, row, filter_columns);
        filter_starts.push_back(filter_columns.size());
      }
    }
    // Smooth, setup.rs:527-573
    double omega = 4.0 / (3.0 * lambda_max);
    Accumulator acc(aggregates, rb * MODES);
    BlockCsr<double> prolongator;
    prolongator.rows = current.rows;
    prolongator.row_block = rb;
    prolongator.col_block = MODES;
    prolongator.starts.push_back(0);
    for (size_t row = 0; row < current.rows; ++row) {
      const uint32_t* nb;
      size_t nn;
      if (filter_starts.empty()) {
        nb = strong_columns.data() + strong_starts[row];
        nn = strong_starts[row + 1] - strong_starts[row];
      } else {
        nb = filter_columns.data() + filter_starts[row];
        nn = filter_starts[row + 1] - filter_starts[row];
      }
      smooth_row(current, tentative, nb, nn, inv, omega, row, acc, prolongator);
    }
    // Product, setup.rs:575-612
    BlockCsr<double> ap;
    ap.rows = current.rows;
    ap.row_block = rb;
    ap.col_block = MODES;
    ap.starts.push_back(0);
    for (size_t row = 0; row < current.rows; ++row) product_row(current, prolongator, row, acc, ap);
    vector<size_t> cstarts;
    vector<std::pair<uint32_t, size_t>> centries;
    prolongator_columns(prolongator, aggregates, cstarts, centries);
    // Galerkin, setup.rs:614-647
    Accumulator acc2(aggregates, MODES * MODES);
    BlockCsr<double> coarse;
    coarse.rows = aggregates;
    coarse.row_block = MODES;
    coarse.col_block = MODES;
    coarse.starts.push_back(0);
    for (size_t c = 0; c < aggregates; ++c) galerkin_row(prolongator, cstarts, centries, ap, c, acc2, coarse);
    // finish_level, setup.rs:650-695
    for (size_t row = 0; row < coarse.rows; ++row)
      for (size_t at = coarse.starts[row]; at < coarse.starts[row + 1]; ++at) {
        if (coarse.columns[at] != row) continue;
        for (size_t d = 0; d < MODES; ++d) {
          double& value = coarse.values[at * 36 + d * MODES + d];
          if (value == 0.0) value = 1.0;
        }
      }
    Level lv;
    lv.a = std::move(current);
    lv.inverse_diagonal = std::move(inv);
    lv.lambda_min = lambda_min;
    lv.lambda_max = lambda_max;
    lv.has_prolongator = true;
    lv.prolongator = std::move(prolongator);
    lv.aggregates = agg->aggregate;
    levels.push_back(std::move(lv));
    current = std::move(coarse);
    near_null = std::move(coarse_null);
    positions = std::move(coarse_positions);
  }
}

// ---------------------------------------------------------------------------------------------
// The V-cycle: crates/solidfem-solve/src/multigrid/cycle.rs, generic over storage S and vector V.
// ---------------------------------------------------------------------------------------------

template <class S>
struct SLevel {
  BlockCsr<S> a;
  vector<S> inv;
  double lambda_min, lambda_max;
  bool has_p;
  BlockCsr<S> p;
  const DenseCholesky* factor;
};

template <class S, class V>
struct Cycle {
  vector<SLevel<S>> levels;
  size_t degree;
  struct Work {
    vector<V> residual, scaled, direction, product, post_rhs, post_x, coarse_rhs, coarse_x;
    vector<double> dense;
    bool parallel;
  };
  vector<Work> work;

  void init() {
    work.resize(levels.size());
    for (size_t i = 0; i < levels.size(); ++i) {
      size_t d = levels[i].a.dofs();
      size_t cd = i + 1 < levels.size() ? levels[i + 1].a.dofs() : 0;
      Work& w = work[i];
      w.residual.assign(d, V(0));
      w.scaled.assign(d, V(0));
      w.direction.assign(d, V(0));
      w.product.assign(d, V(0));
      w.post_rhs.assign(d, V(0));
      w.post_x.assign(d, V(0));
      w.coarse_rhs.assign(cd, V(0));
      w.coarse_x.assign(cd, V(0));
      if (levels[i].factor) w.dense.assign(d, 0.0);
      w.parallel = levels[i].a.values.size() >= MIN_PARALLEL_VALUES;
    }
  }

  // cycle.rs:655-674
  void apply_inverse_diagonal(const SLevel<S>& lv, size_t row, const V* x, V* y) const {
    size_t b = lv.a.row_block;
    const S* d = lv.inv.data() + row * b * b;
    for (size_t p = 0; p < b; ++p) {
      V sum = V(0);
      for (size_t q = 0; q < b; ++q) sum += (V)d[p * b + q] * x[row * b + q];
      y[row * b + p] = sum;
    }
  }

  // cycle.rs:548-564
  void residual(size_t li, const V* b, const V* x, V* r) {
    const SLevel<S>& lv = levels[li];
    size_t rb = lv.a.row_block;
    for_rows(lv.a.rows, work[li].parallel, [&](size_t row) {
      lv.a.multiply_row(row, x, r + row * rb);
      for (size_t p = 0; p < rb; ++p) r[row * rb + p] = b[row * rb + p] - r[row * rb + p];
    });
  }

  // cycle.rs:570-651
  void smooth(size_t li, const V* b, V* x) {
    const SLevel<S>& lv = levels[li];
    Work& w = work[li];
    double theta = 0.5 * (lv.lambda_max + lv.lambda_min);
    double delta = 0.5 * (lv.lambda_max - lv.lambda_min);
    double sigma = theta / delta;
    double rho = 1.0 / sigma;
    size_t block = lv.a.row_block;
    V first = (V)theta;
    V *r = w.residual.data(), *z = w.scaled.data(), *d = w.direction.data(), *ad = w.product.data();
    for_rows(lv.a.rows, w.parallel, [&](size_t row) {
      for (size_t p = 0; p < block; ++p) r[row * block + p] = b[row * block + p];
      apply_inverse_diagonal(lv, row, r, z);
      for (size_t p = 0; p < block; ++p) {
        d[row * block + p] = z[row * block + p] / first;
        x[row * block + p] = d[row * block + p];
      }
    });
    for (size_t s = 1; s < degree; ++s) {
      for_rows(lv.a.rows, w.parallel, [&](size_t row) { lv.a.multiply_row(row, d, ad + row * block); });
      double next_rho = 1.0 / (2.0 * sigma - rho);
      V keep = (V)(next_rho * rho);
      V step = (V)(2.0 * next_rho / delta);
      for_rows(lv.a.rows, w.parallel, [&](size_t row) {
        for (size_t p = 0; p < block; ++p) r[row * block + p] -= ad[row * block + p];
        apply_inverse_diagonal(lv, row, r, z);
        for (size_t p = 0; p < block; ++p) {
          size_t i = row * block + p;
          d[i] = keep * d[i] + step * z[i];
          x[i] += d[i];
        }
      });
      rho = next_rho;
    }
  }

  // cycle.rs:461-539
  void cycle(size_t li, const V* rhs, V* x) {
    const SLevel<S>& lv = levels[li];
    Work& w = work[li];
    if (!lv.has_p) {
      if (lv.factor) {
        size_t n = lv.a.dofs();
        for (size_t i = 0; i < n; ++i) w.dense[i] = (double)rhs[i];
        lv.factor->solve(w.dense.data());
        for (size_t i = 0; i < n; ++i) x[i] = (V)w.dense[i];
      } else {
        smooth(li, rhs, x);
      }
      return;
    }
    smooth(li, rhs, x);
    size_t block = lv.a.row_block;
    residual(li, rhs, x, w.residual.data());
    lv.p.multiply_transpose(w.residual.data(), w.coarse_rhs.data(), w.coarse_rhs.size());
    std::fill(w.coarse_x.begin(), w.coarse_x.end(), V(0));
    cycle(li + 1, w.coarse_rhs.data(), w.coarse_x.data());
    for_rows(lv.a.rows, w.parallel, [&](size_t row) {
      lv.p.multiply_row(row, w.coarse_x.data(), w.product.data() + row * block);
      for (size_t p = 0; p < block; ++p) x[row * block + p] += w.product[row * block + p];
    });
    residual(li, rhs, x, w.post_rhs.data());
    smooth(li, w.post_rhs.data(), w.post_x.data());
    for_rows(lv.a.rows, w.parallel, [&](size_t row) {
      for (size_t p = 0; p < block; ++p) x[row * block + p] += w.post_x[row * block + p];
    });
  }
};

// The finished multigrid in its precision: cycle.rs:254-308 and 430-446.
struct Multigrid {
  int precision = ORC_PRECISION_SINGLE_STORAGE;
  vector<Level> levels;  // f64 setup output, kept for inspection
  Cycle<double, double> dd;
  Cycle<float, double> fd;
  Cycle<float, float> ff;
  vector<float> rhs32, x32;

  template <class S, class V>
  void fill(Cycle<S, V>& c, size_t degree) {
    c.degree = degree;
    c.levels.clear();
    for (auto& lv : levels) {
      SLevel<S> s;
      if constexpr (std::is_same<S, double>::value) {
        s.a = lv.a;
        s.inv = lv.inverse_diagonal;
        if (lv.has_prolongator) s.p = lv.prolongator;
      } else {
        s.a = to_precision<S>(lv.a);
        s.inv.resize(lv.inverse_diagonal.size());
        for (size_t i = 0; i < s.inv.size(); ++i) s.inv[i] = (S)lv.inverse_diagonal[i];
        if (lv.has_prolongator) s.p = to_precision<S>(lv.prolongator);
      }
      s.lambda_min = lv.lambda_min;
      s.lambda_max = lv.lambda_max;
      s.has_p = lv.has_prolongator;
      s.factor = lv.has_factor ? &lv.factor : nullptr;
      c.levels.push_back(std::move(s));
    }
    c.init();
  }

  void finish(size_t degree) {
    if (precision == ORC_PRECISION_DOUBLE)
      fill(dd, degree);
    else if (precision == ORC_PRECISION_SINGLE_STORAGE)
      fill(fd, degree);
    else {
      fill(ff, degree);
      rhs32.assign(levels[0].a.dofs(), 0.0f);
      x32.assign(levels[0].a.dofs(), 0.0f);
    }
  }

  void apply(const double* r, double* out) {
    if (precision == ORC_PRECISION_DOUBLE)
      dd.cycle(0, r, out);
    else if (precision == ORC_PRECISION_SINGLE_STORAGE)
      fd.cycle(0, r, out);
    else {
      size_t n = rhs32.size();
      for (size_t i = 0; i < n; ++i) rhs32[i] = (float)r[i];
      ff.cycle(0, rhs32.data(), x32.data());
      for (size_t i = 0; i < n; ++i) out[i] = (double)x32[i];
    }
  }

  // mod.rs:186-195 and cycle.rs:676-698
  void stats(orc_mg_stats* st) const {
    size_t s_bytes = precision == ORC_PRECISION_DOUBLE ? 8 : 4;
    double finest = levels.empty() ? 1.0 : (double)levels[0].a.values.size();
    size_t stored = 0, memory = 0;
    for (auto& lv : levels) {
      stored += lv.a.values.size();
      memory += lv.a.starts.size() * 8 + lv.a.columns.size() * 4 + lv.a.values.size() * s_bytes;
      memory += lv.inverse_diagonal.size() * s_bytes;
      if (lv.has_prolongator)
        memory += lv.prolongator.starts.size() * 8 + lv.prolongator.columns.size() * 4 +
                  lv.prolongator.values.size() * s_bytes;
      if (lv.has_factor) memory += lv.factor.factor.size() * 8;
    }
    st->levels = levels.size();
    st->coarse_dofs = levels.empty() ? 0 : levels.back().a.dofs();
    st->operator_complexity = (double)stored / finest;
    st->memory_bytes = memory;
  }
};

// ---------------------------------------------------------------------------------------------
// PCG: crates/solidfem-solve/src/pcg.rs. Jacobi: crates/solidfem-solve/src/preconditioner.rs.
// ---------------------------------------------------------------------------------------------

static double dot(const double* a, const double* b, size_t n) {
  double sum = 0.0;
  for (size_t i = 0; i < n; ++i) sum += a[i] * b[i];
  return sum;
}
static double norm(const double* a, size_t n) { return std::sqrt(dot(a, a, n)); }

struct Pcg {
  const Csr* matrix = nullptr;
  std::function<void(const double*, double*)> precondition;
  vector<double> rhs, x, r, z, p, ap;
  double rz = 0, rhs_norm = 0, relative_residual = 0;
  uint64_t iterations = 0, max_iterations = 0;
  double tolerance = 1e-9;
  bool floor_reached = false;
  int status = ORC_ACTIVE;
  uint64_t fail_iteration = 0;
  double fail_curvature = 0;
  bool parallel = false;

  void system_multiply(const double* in, double* out) {
    const Csr& m = *matrix;
    for_rows(m.size, parallel, [&](size_t row) { m.multiply_rows(row, row + 1, in, out + row); });
  }

  void init(const Csr* m, vector<double> b, double tol, uint64_t max_it) {
    matrix = m;
    size_t n = m->size;
    rhs_norm = norm(b.data(), b.size());
    max_iterations = max_it ? max_it : 10 * (uint64_t)n + 1000;
    r = b;
    rhs = std::move(b);
    x.assign(n, 0.0);
    z.assign(n, 0.0);
    p.assign(n, 0.0);
    ap.assign(n, 0.0);
    tolerance = tol;
    parallel = m->columns.size() >= MIN_PARALLEL_VALUES;
    if (rhs_norm == 0.0) {
      status = ORC_CONVERGED;
    } else {
      reset_direction();
      relative_residual = 1.0;
    }
  }
  void reset_direction() {
    precondition(r.data(), z.data());
    p = z;
    rz = dot(r.data(), z.data(), r.size());
  }
  // pcg.rs:216-275. Returns the status after the iteration.
  int iterate() {
    size_t n = rhs.size();
    system_multiply(p.data(), ap.data());
    double curvature = dot(p.data(), ap.data(), n);
    if (std::isnan(curvature) || curvature <= 0.0 || !std::isfinite(rz)) {
      status = ORC_FAILED_NOT_POSITIVE_DEFINITE;
      fail_iteration = iterations;
      fail_curvature = curvature;
      return status;
    }
    double alpha = rz / curvature;
    for (size_t i = 0; i < n; ++i) x[i] += alpha * p[i];
    double na = -alpha;
    for (size_t i = 0; i < n; ++i) r[i] += na * ap[i];
    iterations += 1;
    relative_residual = norm(r.data(), n) / rhs_norm;
    if (relative_residual <= tolerance) {
      vector<double> residual(n);
      system_multiply(x.data(), residual.data());
      for (size_t i = 0; i < n; ++i) residual[i] = rhs[i] - residual[i];
      relative_residual = norm(residual.data(), n) / rhs_norm;
      double floor = matrix->multiply_rounding_bound(x.data()) / rhs_norm;
      floor_reached = relative_residual > tolerance && relative_residual <= floor;
      if (relative_residual <= tolerance || floor_reached) {
        status = ORC_CONVERGED;
        return status;
      }
      r = residual;
      reset_direction();
    } else {
      precondition(r.data(), z.data());
      double rz_next = dot(r.data(), z.data(), n);
      double beta = rz_next / rz;
      rz = rz_next;
      for (size_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
    if (iterations >= max_iterations) {
      status = ORC_FAILED_NOT_CONVERGED;
      return status;
    }
    return ORC_ACTIVE;
  }
};

// ---------------------------------------------------------------------------------------------
// Loads, rigid modes, constraint check: crates/solidfem-elastic/src/{loads,rigid_modes,
// constraints}.rs
// ---------------------------------------------------------------------------------------------

// loads.rs:174-201
static void triangle_shape(double r, double s, double v[6], double dr[6], double ds[6]) {
  double l1 = 1.0 - r - s;
  v[0] = l1 * (2.0 * l1 - 1.0);
  v[1] = r * (2.0 * r - 1.0);
  v[2] = s * (2.0 * s - 1.0);
  v[3] = 4.0 * l1 * r;
  v[4] = 4.0 * r * s;
  v[5] = 4.0 * s * l1;
  dr[0] = -(4.0 * l1 - 1.0);
  dr[1] = 4.0 * r - 1.0;
  dr[2] = 0.0;
  dr[3] = 4.0 * (l1 - r);
  dr[4] = 4.0 * s;
  dr[5] = -4.0 * s;
  ds[0] = -(4.0 * l1 - 1.0);
  ds[1] = 0.0;
  ds[2] = 4.0 * s - 1.0;
  ds[3] = -4.0 * r;
  ds[4] = 4.0 * r;
  ds[5] = 4.0 * (l1 - s);
}

// loads.rs:10-41
static void add_traction(const QuadMesh& q, const array<uint32_t, 6>& face, const double t[3],
                         vector<double>& load) {
  P3 pos[6];
  for (int i = 0; i < 6; ++i) pos[i] = q.nodes[face[i]];
  for (int pt = 0; pt < 6; ++pt) {
    double r = TRIANGLE[pt][0], s = TRIANGLE[pt][1], weight = TRIANGLE[pt][2];
    double v[6], dr[6], ds[6];
    triangle_shape(r, s, v, dr, ds);
    double tr[3] = {0, 0, 0}, ts[3] = {0, 0, 0};
    for (int nd = 0; nd < 6; ++nd)
      for (int ax = 0; ax < 3; ++ax) {
        tr[ax] += dr[nd] * pos[nd][ax];
        ts[ax] += ds[nd] * pos[nd][ax];
      }
    double nrm[3] = {tr[1] * ts[2] - tr[2] * ts[1], tr[2] * ts[0] - tr[0] * ts[2],
                     tr[0] * ts[1] - tr[1] * ts[0]};
    double length = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
    double measure = 0.5 * length * weight;
    for (int nd = 0; nd < 6; ++nd)
      for (int ax = 0; ax < 3; ++ax) load[3 * (size_t)face[nd] + ax] += t[ax] * v[nd] * measure;
  }
}

// rigid_modes.rs:36-83
static vector<double> free_rigid_body_modes(const vector<P3>& nodes, const vector<uint32_t>& free,
                                            size_t free_count) {
  double c[3] = {0, 0, 0};
  for (size_t n = 0; n < nodes.size(); ++n)
    if (free[n] != FIXED)
      for (int a = 0; a < 3; ++a) c[a] += nodes[n][a];
  double divisor = (double)std::max<size_t>(free_count, 1);
  for (int a = 0; a < 3; ++a) c[a] /= divisor;
  double reach = 0.0;
  for (size_t n = 0; n < nodes.size(); ++n)
    if (free[n] != FIXED)
      for (int a = 0; a < 3; ++a) reach = std::max(reach, std::fabs(nodes[n][a] - c[a]));
  double scale = reach > 0.0 ? 1.0 / reach : 1.0;
  vector<double> modes(3 * free_count * 6, 0.0);
  for (size_t n = 0; n < nodes.size(); ++n) {
    if (free[n] == FIXED) continue;
    size_t at = 3 * (size_t)free[n] * 6;
    double x = (nodes[n][0] - c[0]) * scale;
    double y = (nodes[n][1] - c[1]) * scale;
    double z = (nodes[n][2] - c[2]) * scale;
    double rows[3][6] = {{1, 0, 0, 0, z, -y}, {0, 1, 0, -z, 0, x}, {0, 0, 1, y, -x, 0}};
    for (int r = 0; r < 3; ++r)
      for (int k = 0; k < 6; ++k) modes[at + r * 6 + k] = rows[r][k];
  }
  return modes;
}

static double distance3(const P3& a, const P3& b) {
  double d[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
  return std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
}

// constraints.rs:40-73. Returns true when the points hold the body.
static bool points_hold(const vector<P3>& pts, double size) {
  if (pts.empty()) return false;
  double limit = 1e-9 * size;
  P3 first = pts[0], far = first;
  double far_d = 0.0;
  for (auto& p : pts) {
    double d = distance3(first, p);
    if (d > far_d) {
      far = p;
      far_d = d;
    }
  }
  if (far_d <= limit) return false;
  double axis[3] = {(far[0] - first[0]) / far_d, (far[1] - first[1]) / far_d, (far[2] - first[2]) / far_d};
  for (auto& p : pts) {
    double v[3] = {p[0] - first[0], p[1] - first[1], p[2] - first[2]};
    double along = v[0] * axis[0] + v[1] * axis[1] + v[2] * axis[2];
    double off[3] = {v[0] - along * axis[0], v[1] - along * axis[1], v[2] - along * axis[2]};
    if (std::sqrt(off[0] * off[0] + off[1] * off[1] + off[2] * off[2]) > limit) return true;
  }
  return false;
}

// constraints.rs:81-135
static int check_constraints(const QuadMesh& q, const vector<char>& fixed) {
  bool any = false;
  for (char f : fixed) any = any || f;
  if (!any) return ORC_NO_FIXED_NODES;
  auto bodies = face_connected_bodies(q);
  vector<vector<uint32_t>> body_nodes;
  vector<double> sizes;
  for (auto& tets : bodies) {
    vector<uint32_t> nodes;
    for (uint32_t t : tets)
      for (uint32_t n : q.tets[t]) nodes.push_back(n);
    std::sort(nodes.begin(), nodes.end());
    nodes.erase(std::unique(nodes.begin(), nodes.end()), nodes.end());
    P3 lo = {INFINITY, INFINITY, INFINITY}, hi = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t n : nodes)
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::min(lo[a], q.nodes[n][a]);
        hi[a] = std::max(hi[a], q.nodes[n][a]);
      }
    sizes.push_back(distance3(lo, hi));
    body_nodes.push_back(std::move(nodes));
  }
  vector<char> held = fixed;
  vector<char> anchored(bodies.size(), 0);
  while (true) {
    bool changed = false;
    for (size_t b = 0; b < bodies.size(); ++b) {
      if (anchored[b]) continue;
      vector<P3> pts;
      for (uint32_t n : body_nodes[b])
        if (held[n]) pts.push_back(q.nodes[n]);
      if (points_hold(pts, sizes[b])) {
        anchored[b] = 1;
        changed = true;
        for (uint32_t n : body_nodes[b]) held[n] = 1;
      }
    }
    if (!changed) break;
  }
  for (size_t b = 0; b < bodies.size(); ++b)
    if (!anchored[b]) return ORC_BODY_NOT_HELD;
  return 0;
}

// ---------------------------------------------------------------------------------------------
// Recovery: crates/solidfem-elastic/src/{results,patch}.rs
// ---------------------------------------------------------------------------------------------

struct PatchFit {
  double centre[3];
  double scale;
  double coefficients[4][6];
  void offsets(const double* p, double t[4]) const {
    t[0] = 1.0;
    t[1] = (p[0] - centre[0]) / scale;
    t[2] = (p[1] - centre[1]) / scale;
    t[3] = (p[2] - centre[2]) / scale;
  }
  // patch.rs:69-78
  void at(const double* p, double out[6]) const {
    double t[4];
    offsets(p, t);
    for (int k = 0; k < 6; ++k) out[k] = 0.0;
    for (int term = 0; term < 4; ++term)
      for (int k = 0; k < 6; ++k) out[k] += t[term] * coefficients[term][k];
  }
};

// patch.rs:83-120
static bool patch_solve(double m[4][4], double rhs[4][6]) {
  for (int c = 0; c < 4; ++c) {
    int pivot = c;
    for (int r = c + 1; r < 4; ++r)
      if (std::fabs(m[r][c]) > std::fabs(m[pivot][c])) pivot = r;
    if (std::fabs(m[pivot][c]) <= 1e-12) return false;
    for (int k = 0; k < 4; ++k) std::swap(m[c][k], m[pivot][k]);
    for (int k = 0; k < 6; ++k) std::swap(rhs[c][k], rhs[pivot][k]);
    double prow[4], prhs[6];
    for (int k = 0; k < 4; ++k) prow[k] = m[c][k];
    for (int k = 0; k < 6; ++k) prhs[k] = rhs[c][k];
    for (int r = c + 1; r < 4; ++r) {
      double factor = m[r][c] / prow[c];
      for (int k = c; k < 4; ++k) m[r][k] -= factor * prow[k];
      for (int k = 0; k < 6; ++k) rhs[r][k] -= factor * prhs[k];
    }
  }
  for (int c = 3; c >= 0; --c) {
    double value[6];
    for (int k = 0; k < 6; ++k) value[k] = rhs[c][k];
    for (int j = c + 1; j < 4; ++j)
      for (int k = 0; k < 6; ++k) value[k] -= m[c][j] * rhs[j][k];
    for (int k = 0; k < 6; ++k) rhs[c][k] = value[k] / m[c][c];
  }
  return true;
}

// patch.rs:37-66
static bool patch_fit(const P3& centre, const vector<std::pair<P3, array<double, 6>>>& samples,
                      PatchFit& fit) {
  double scale = 0.0;
  for (auto& s : samples)
    for (int a = 0; a < 3; ++a) scale = std::max(scale, std::fabs(s.first[a] - centre[a]));
  if (samples.empty() || scale == 0.0) return false;
  for (int a = 0; a < 3; ++a) fit.centre[a] = centre[a];
  fit.scale = scale;
  double m[4][4] = {{0}}, rhs[4][6] = {{0}};
  for (auto& s : samples) {
    double t[4];
    fit.offsets(s.first.data(), t);
    for (int i = 0; i < 4; ++i) {
      for (int j = 0; j < 4; ++j) m[i][j] += t[i] * t[j];
      for (int k = 0; k < 6; ++k) rhs[i][k] += t[i] * s.second[k];
    }
  }
  if (!patch_solve(m, rhs)) return false;
  for (int i = 0; i < 4; ++i)
    for (int k = 0; k < 6; ++k) fit.coefficients[i][k] = rhs[i][k];
  return true;
}

// results.rs:555-569
static int nearest_natural_point(const QPoint* pts, int count, const double node[3]) {
  double best = std::numeric_limits<double>::max();
  int index = 0;
  for (int i = 0; i < count; ++i) {
    double d = 0.0;
    for (int a = 0; a < 3; ++a) d = d + (pts[i].natural[a] - node[a]) * (pts[i].natural[a] - node[a]);
    if (d < best) {
      best = d;
      index = i;
    }
  }
  return index;
}

struct Recovered {
  vector<orc_point_stress> points;
  vector<array<double, 6>> nodal_stress;
  vector<double> nodal_von_mises;
};

// results.rs:470-539 (elements, then vertex fits) and 376-410 (the field).
static int recover(const QuadMesh& q, const MaterialField& field, int quadrature,
                   const vector<P3>& disp, Recovered& out) {
  const QPoint* pts;
  int count;
  rule_points(quadrature, &pts, &count);
  int nearest[10];
  for (int n = 0; n < 10; ++n) nearest[n] = nearest_natural_point(pts, count, NODE_NATURAL[n]);
  size_t node_count = q.nodes.size();
  vector<Material> point_materials;
  out.points.clear();
  out.points.reserve(q.tets.size() * count);
  vector<std::pair<array<double, 6>, double>> worst(node_count, {{0, 0, 0, 0, 0, 0}, -std::numeric_limits<double>::max()});
  for (size_t t = 0; t < q.tets.size(); ++t) {
    P3 nodes[10];
    double u[10][3];
    for (int a = 0; a < 10; ++a) {
      nodes[a] = q.nodes[q.tets[t][a]];
      for (int k = 0; k < 3; ++k) u[a][k] = disp[q.tets[t][a]][k];
    }
    for (int qi = 0; qi < count; ++qi) {
      Geometry g;
      if (!point_geometry(nodes, pts[qi].natural, g)) return ORC_ELEMENT_INVERTED;
      Material m = field.at(g.position);
      if (!m.valid()) return ORC_ELEMENT_MATERIAL;
      double e[6], s[6];
      strain_at(g, u, e);
      stress_at(m, e, s);
      orc_point_stress ps;
      ps.tet = (uint32_t)t;
      ps.point = (uint32_t)qi;
      for (int a = 0; a < 3; ++a) ps.position[a] = g.position[a];
      for (int k = 0; k < 6; ++k) ps.stress[k] = s[k];
      ps.von_mises = von_mises(s);
      out.points.push_back(ps);
      point_materials.push_back(m);
    }
    const Material* em = point_materials.data() + point_materials.size() - count;
    for (int n = 0; n < 10; ++n) {
      Geometry g;
      if (!point_geometry(nodes, NODE_NATURAL[n], g)) return ORC_ELEMENT_INVERTED;
      Material m = em[nearest[n]];
      double e[6], s[6];
      strain_at(g, u, e);
      stress_at(m, e, s);
      double vm = von_mises(s);
      auto& w = worst[q.tets[t][n]];
      if (vm > w.second) {
        for (int k = 0; k < 6; ++k) w.first[k] = s[k];
        w.second = vm;
      }
    }
  }
  // build_patches, results.rs:414-435
  size_t vertices = q.vertex_count;
  vector<size_t> offsets(vertices + 1, 0);
  for (auto& t : q.tets)
    for (int c = 0; c < 4; ++c) offsets[t[c] + 1] += 1;
  for (size_t i = 1; i < offsets.size(); ++i) offsets[i] += offsets[i - 1];
  vector<size_t> next = offsets;
  vector<uint32_t> incident(offsets[vertices]);
  for (size_t t = 0; t < q.tets.size(); ++t)
    for (int c = 0; c < 4; ++c) incident[next[q.tets[t][c]]++] = (uint32_t)t;
  // fit_next_vertex, results.rs:438-466
  vector<PatchFit> fits(vertices);
  vector<char> has_fit(vertices, 0);
  for (size_t v = 0; v < vertices; ++v) {
    vector<std::pair<P3, array<double, 6>>> samples;
    bool uniform = true;
    bool have_first = false;
    Material first{0, 0};
    for (size_t k = offsets[v]; k < offsets[v + 1]; ++k) {
      size_t start = (size_t)incident[k] * count;
      for (size_t p = start; p < start + (size_t)count; ++p) {
        const Material& m = point_materials[p];
        if (!have_first) {
          first = m;
          have_first = true;
        } else if (std::memcmp(&first.E, &m.E, 8) != 0 || std::memcmp(&first.nu, &m.nu, 8) != 0) {
          uniform = false;
        }
        P3 pos = {out.points[p].position[0], out.points[p].position[1], out.points[p].position[2]};
        array<double, 6> st;
        for (int c = 0; c < 6; ++c) st[c] = out.points[p].stress[c];
        samples.push_back({pos, st});
      }
    }
    if (uniform) has_fit[v] = patch_fit(q.nodes[v], samples, fits[v]) ? 1 : 0;
  }
  // into_field, results.rs:376-410
  out.nodal_stress.assign(node_count, {0, 0, 0, 0, 0, 0});
  for (size_t v = 0; v < vertices; ++v) {
    if (has_fit[v]) {
      double s[6];
      fits[v].at(q.nodes[v].data(), s);
      for (int k = 0; k < 6; ++k) out.nodal_stress[v][k] = s[k];
    } else {
      out.nodal_stress[v] = worst[v].first;
    }
  }
  vector<char> done(node_count - vertices, 0);
  for (auto& t : q.tets)
    for (int e = 0; e < 6; ++e) {
      size_t mid = t[4 + e];
      if (done[mid - vertices]) continue;
      done[mid - vertices] = 1;
      uint32_t a = t[EDGE_CORNERS[e][0]], b = t[EDGE_CORNERS[e][1]];
      if (has_fit[a] && has_fit[b]) {
        double p[6], r[6];
        fits[a].at(q.nodes[mid].data(), p);
        fits[b].at(q.nodes[mid].data(), r);
        for (int k = 0; k < 6; ++k) out.nodal_stress[mid][k] = 0.5 * (p[k] + r[k]);
      } else {
        out.nodal_stress[mid] = worst[mid].first;
      }
    }
  out.nodal_von_mises.resize(node_count);
  for (size_t n = 0; n < node_count; ++n) out.nodal_von_mises[n] = von_mises(out.nodal_stress[n].data());
  return 0;
}

}  // namespace orc

// =============================================================================================
// The C interface the tests and the CPU baseline call through ctypes.
// =============================================================================================

using namespace orc;

struct orc_mesh {
  QuadMesh q;
  vector<BoundaryFace> faces;
};

struct orc_study {
  const orc_mesh* mesh = nullptr;
  MaterialField field;
  int quadrature = 0;
  vector<uint32_t> free;
  size_t free_count = 0;
  vector<double> load, rhs;
  Csr matrix;
  Multigrid mg;
  vector<double> jacobi;
  bool use_mg = false;
  Pcg pcg;
  SetupError setup_error;
  double seconds[4] = {0, 0, 0, 0};
  Recovered recovered;
  bool recovered_done = false;
  vector<std::pair<size_t, double>> prescribed;           // (free dof, value), ascending dof
  vector<std::array<double, 3>> prescribed_nodes;         // (node, axis, value) as doubles
};

// StudyBuilder::apply_prescribed (study.rs:564-593): each prescribed component in ascending
// order moves what it forces on the unconstrained unknowns to the right-hand side, and its row
// and column are emptied but for the diagonal; its right-hand side becomes diagonal x value.
static void apply_prescribed(Csr& m, vector<double>& rhs, const vector<std::pair<size_t, double>>& prescribed) {
  vector<char> constrained(rhs.size(), 0);
  for (auto& p : prescribed) constrained[p.first] = 1;
  for (auto& p : prescribed) {
    size_t dof = p.first;
    double value = p.second;
    vector<std::pair<uint32_t, double>> entries;
    for (size_t at = m.row_starts[dof]; at < m.row_starts[dof + 1]; ++at)
      if (m.columns[at] != dof) entries.push_back({m.columns[at], m.values[at]});
    for (auto& e : entries) {
      size_t c = e.first;
      if (!constrained[c]) rhs[c] -= e.second * value;
      m.add(c, (uint32_t)dof, -e.second);
      m.add(dof, e.first, -e.second);
    }
  }
  for (auto& p : prescribed) rhs[p.first] = m.get(p.first, (uint32_t)p.first) * p.second;
}

extern "C" {

int orc_box_mesh(const double origin[3], const double size[3], const uint64_t divisions[3],
                 orc_mesh** out) {
  size_t div[3] = {(size_t)divisions[0], (size_t)divisions[1], (size_t)divisions[2]};
  TetMesh lin;
  int code = box_tet_mesh(origin, size, div, lin);
  if (code) return code;
  orc_mesh* m = new orc_mesh;
  m->q = from_linear(lin);
  m->faces = boundary_faces(m->q);
  *out = m;
  return 0;
}

int orc_linear_mesh(const double* positions, uint64_t n, const uint32_t* tets, uint64_t ntets,
                    orc_mesh** out) {
  TetMesh lin;
  lin.positions.resize(n);
  for (uint64_t i = 0; i < n; ++i) lin.positions[i] = {positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]};
  lin.tets.resize(ntets);
  for (uint64_t t = 0; t < ntets; ++t)
    for (int k = 0; k < 4; ++k) lin.tets[t][k] = tets[4 * t + k];
  int code = validate_mesh(lin);
  if (code) return code;
  orc_mesh* m = new orc_mesh;
  m->q = from_linear(lin);
  m->faces = boundary_faces(m->q);
  *out = m;
  return 0;
}

void orc_mesh_free(orc_mesh* m) { delete m; }
uint64_t orc_mesh_node_count(const orc_mesh* m) { return m->q.nodes.size(); }
uint64_t orc_mesh_tet_count(const orc_mesh* m) { return m->q.tets.size(); }
uint64_t orc_mesh_vertex_count(const orc_mesh* m) { return m->q.vertex_count; }
uint64_t orc_mesh_face_count(const orc_mesh* m) { return m->faces.size(); }
void orc_mesh_nodes(const orc_mesh* m, double* out) {
  for (size_t i = 0; i < m->q.nodes.size(); ++i)
    for (int a = 0; a < 3; ++a) out[3 * i + a] = m->q.nodes[i][a];
}
void orc_mesh_tets(const orc_mesh* m, uint32_t* out) {
  for (size_t t = 0; t < m->q.tets.size(); ++t)
    for (int k = 0; k < 10; ++k) out[10 * t + k] = m->q.tets[t][k];
}
void orc_mesh_faces(const orc_mesh* m, orc_face* out) {
  for (size_t i = 0; i < m->faces.size(); ++i) {
    out[i].tet = m->faces[i].tet;
    out[i].face = m->faces[i].face;
    for (int k = 0; k < 6; ++k) out[i].nodes[k] = m->faces[i].nodes[k];
  }
}

void orc_set_threads(int threads) { g_threads = threads < 1 ? 1 : threads; }

int orc_default_threads(void) {
#ifdef _OPENMP
  int logical = omp_get_num_procs();
#else
  int logical = 1;
#endif
  int t = logical / 2;
  return t < 1 ? 1 : (t > 8 ? 8 : t);
}

static double now_seconds() {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

// StudyBuilder::new + step + finish (study.rs:419-656) in one call.
int orc_study_new_prescribed(const orc_mesh* mesh, const orc_material* material, const orc_options* options,
                             const uint32_t* fixed_nodes, uint64_t n_fixed, const orc_nodal_force* forces,
                             uint64_t n_forces, const orc_face* faces, const double* tractions,
                             uint64_t n_tractions, const orc_prescribed* prescribed, uint64_t n_prescribed,
                             orc_study** out);

int orc_study_new(const orc_mesh* mesh, const orc_material* material, const orc_options* options,
                  const uint32_t* fixed_nodes, uint64_t n_fixed, const orc_nodal_force* forces,
                  uint64_t n_forces, const orc_face* faces, const double* tractions,
                  uint64_t n_tractions, orc_study** out) {
  return orc_study_new_prescribed(mesh, material, options, fixed_nodes, n_fixed, forces, n_forces, faces, tractions,
                                  n_tractions, nullptr, 0, out);
}

// With prescribed components the reference checks the held DOFs' rank instead of the fixed
// nodes (constraints.rs:162-256); the oracle leaves that refusal to the product's tests and
// takes the model as held.
int orc_study_new_prescribed(const orc_mesh* mesh, const orc_material* material, const orc_options* options,
                             const uint32_t* fixed_nodes, uint64_t n_fixed, const orc_nodal_force* forces,
                             uint64_t n_forces, const orc_face* faces, const double* tractions,
                             uint64_t n_tractions, const orc_prescribed* prescribed, uint64_t n_prescribed,
                             orc_study** out) {
  double t0 = now_seconds();
  const QuadMesh& q = mesh->q;
  size_t node_count = q.nodes.size();
  vector<char> is_fixed(node_count, 0);
  for (uint64_t i = 0; i < n_fixed; ++i) {
    if (fixed_nodes[i] >= node_count) return ORC_NODE_RANGE;
    is_fixed[fixed_nodes[i]] = 1;
  }
  if (n_prescribed == 0)
    if (int c = check_constraints(q, is_fixed)) return c;
  // build_load, study.rs:696-735
  vector<double> load(3 * node_count, 0.0);
  for (uint64_t i = 0; i < n_forces; ++i) {
    if (forces[i].node >= node_count) return ORC_NODE_RANGE;
    for (int a = 0; a < 3; ++a)
      if (!std::isfinite(forces[i].force[a])) return ORC_NONFINITE_LOAD;
    for (int a = 0; a < 3; ++a) load[3 * (size_t)forces[i].node + a] += forces[i].force[a];
  }
  if (n_tractions) {
    for (uint64_t i = 0; i < n_tractions; ++i) {
      bool on = false;
      for (auto& bf : mesh->faces)
        if (bf.tet == faces[i].tet && bf.face == faces[i].face) {
          on = true;
          for (int k = 0; k < 6; ++k) on = on && bf.nodes[k] == faces[i].nodes[k];
          break;
        }
      if (!on) return ORC_FACE_NOT_ON_BOUNDARY;
      for (int a = 0; a < 3; ++a)
        if (!std::isfinite(tractions[3 * i + a])) return ORC_NONFINITE_LOAD;
      array<uint32_t, 6> fn;
      for (int k = 0; k < 6; ++k) fn[k] = faces[i].nodes[k];
      add_traction(q, fn, tractions + 3 * i, load);
    }
  }
  orc_study* s = new orc_study;
  s->mesh = mesh;
  s->field.spec = *material;
  s->quadrature = options->quadrature;
  s->free.assign(node_count, FIXED);
  for (size_t n = 0; n < node_count; ++n)
    if (!is_fixed[n]) s->free[n] = (uint32_t)s->free_count++;
  for (size_t n = 0; n < node_count; ++n)
    if (s->free[n] != FIXED)
      for (int a = 0; a < 3; ++a) s->rhs.push_back(load[3 * n + a]);
  // prescribed_dofs, study.rs:659-680
  for (uint64_t i = 0; i < n_prescribed; ++i) {
    const orc_prescribed& p = prescribed[i];
    if (p.axis > 2 || !std::isfinite(p.value) || p.node >= node_count || s->free[p.node] == FIXED) {
      delete s;
      return ORC_BAD_PRESCRIBED;
    }
    s->prescribed.push_back({3 * (size_t)s->free[p.node] + p.axis, p.value});
    s->prescribed_nodes.push_back({(double)p.node, (double)p.axis, p.value});
  }
  std::sort(s->prescribed.begin(), s->prescribed.end());
  bool all_zero = true;
  for (double v : s->rhs) all_zero = all_zero && v == 0.0;
  for (auto& p : s->prescribed) all_zero = all_zero && p.second == 0.0;
  if (all_zero) {
    delete s;
    return ORC_NO_EFFECTIVE_LOAD;
  }
  // free_stiffness_pattern, assembly.rs:55-81
  vector<vector<uint32_t>> mapped(q.tets.size());
  for (size_t t = 0; t < q.tets.size(); ++t)
    for (uint32_t nd : q.tets[t])
      if (s->free[nd] != FIXED) mapped[t].push_back(s->free[nd]);
  s->matrix = Csr::from_block_connectivity(s->free_count, 3, mapped);
  // add_element_stiffness, assembly.rs:87-130
  double ke[900];
  for (size_t t = 0; t < q.tets.size(); ++t) {
    P3 nodes[10];
    for (int a = 0; a < 10; ++a) nodes[a] = q.nodes[q.tets[t][a]];
    if (int c = element_stiffness(nodes, s->field, s->quadrature, ke)) {
      delete s;
      return c;
    }
    for (int a = 0; a < 10; ++a) {
      uint32_t rf = s->free[q.tets[t][a]];
      if (rf == FIXED) continue;
      for (int b = 0; b < 10; ++b) {
        uint32_t cf = s->free[q.tets[t][b]];
        if (cf == FIXED) continue;
        for (int i = 0; i < 3; ++i)
          for (int k = 0; k < 3; ++k)
            s->matrix.add(3 * (size_t)rf + i, (uint32_t)(3 * (size_t)cf + k), ke[(3 * a + i) * 30 + (3 * b + k)]);
      }
    }
  }
  if (!s->prescribed.empty()) apply_prescribed(s->matrix, s->rhs, s->prescribed);
  double t1 = now_seconds();
  s->seconds[0] = t1 - t0;
  s->use_mg = options->preconditioner == ORC_PRECONDITIONER_MULTIGRID;
  if (s->use_mg) {
    vector<double> modes = free_rigid_body_modes(q.nodes, s->free, s->free_count);
    for (auto& p : s->prescribed) std::fill(modes.begin() + p.first * 6, modes.begin() + p.first * 6 + 6, 0.0);
    vector<P3> positions;
    for (size_t n = 0; n < node_count; ++n)
      if (s->free[n] != FIXED) positions.push_back(q.nodes[n]);
    MgOptions mo;
    mo.reach = options->neighbour_reach;
    mo.coarse_dofs = options->coarse_dofs;
    mo.max_levels = options->max_levels;
    mo.degree = options->smoother_degree;
    mo.range = options->smoother_range;
    mo.precision = options->precision;
    s->mg.precision = options->precision;
    if (!build_hierarchy(s->matrix, modes, positions, mo, s->mg.levels, s->setup_error)) {
      int c = s->setup_error.code;
      delete s;
      return c;
    }
    s->mg.finish(mo.degree);
    orc_study* self = s;
    s->pcg.precondition = [self](const double* r, double* z) { self->mg.apply(r, z); };
  } else {
    // preconditioner.rs:221-234
    vector<double> diag(s->matrix.size);
    for (size_t i = 0; i < s->matrix.size; ++i) {
      double v = s->matrix.get(i, (uint32_t)i);
      if (std::isnan(v) || v <= 0.0 || !std::isfinite(v)) {
        delete s;
        return ORC_JACOBI_DIAGONAL;
      }
      diag[i] = 1.0 / v;
    }
    s->jacobi = diag;
    orc_study* self = s;
    s->pcg.precondition = [self](const double* r, double* z) {
      for (size_t i = 0; i < self->jacobi.size(); ++i) z[i] = r[i] * self->jacobi[i];
    };
  }
  double t2 = now_seconds();
  s->seconds[1] = t2 - t1;
  s->pcg.init(&s->matrix, s->rhs, options->tolerance, options->max_iterations);
  s->seconds[0] += now_seconds() - t2;
  *out = s;
  return 0;
}

void orc_study_free(orc_study* s) { delete s; }

// StaticStudy::step, study.rs:202-215 (no cancel: the oracle runs uninterrupted).
int orc_study_step(orc_study* s, uint64_t max_iterations, orc_progress* progress) {
  double t0 = now_seconds();
  for (uint64_t i = 0; i < max_iterations && s->pcg.status == ORC_ACTIVE; ++i) s->pcg.iterate();
  s->seconds[2] += now_seconds() - t0;
  progress->iteration = s->pcg.iterations;
  progress->relative_residual = s->pcg.relative_residual;
  progress->at_rounding_floor = s->pcg.floor_reached ? 1 : 0;
  progress->status = s->pcg.status;
  progress->fail_curvature = s->pcg.fail_curvature;
  return s->pcg.status;
}

// StaticStudy::displacements, study.rs:219-238: every mesh node, zero at fixed nodes.
void orc_study_displacements(const orc_study* s, double* out) {
  const vector<double>& x = s->pcg.x;
  for (size_t n = 0; n < s->free.size(); ++n)
    for (int a = 0; a < 3; ++a)
      out[3 * n + a] = s->free[n] == FIXED ? 0.0 : x[3 * (size_t)s->free[n] + a];
  // A prescribed component is exact, not the solver's estimate of it (study.rs:233-236).
  for (auto& p : s->prescribed_nodes) out[3 * (size_t)p[0] + (size_t)p[1]] = p[2];
}

// FNV-1a over the displacement bits, crates/solidfem/tests/validation/multigrid_precision.rs:216-226.
uint64_t orc_study_fingerprint(const orc_study* s) {
  vector<double> d(3 * s->free.size());
  orc_study_displacements(s, d.data());
  uint64_t hash = 0xcbf29ce484222325ull;
  for (double v : d) {
    uint64_t bits;
    std::memcpy(&bits, &v, 8);
    for (int b = 0; b < 8; ++b) {
      hash ^= (bits >> (8 * b)) & 0xff;
      hash *= 0x00000100000001b3ull;
    }
  }
  return hash;
}

void orc_study_seconds(const orc_study* s, double out[4]) {
  for (int i = 0; i < 4; ++i) out[i] = s->seconds[i];
}

uint64_t orc_study_free_dofs(const orc_study* s) { return s->matrix.size; }
uint64_t orc_study_nonzeros(const orc_study* s) { return s->matrix.columns.size(); }
void orc_study_rhs(const orc_study* s, double* out) { std::memcpy(out, s->rhs.data(), s->rhs.size() * 8); }
void orc_study_matrix(const orc_study* s, uint64_t* row_starts, uint32_t* columns, double* values) {
  for (size_t i = 0; i <= s->matrix.size; ++i) row_starts[i] = s->matrix.row_starts[i];
  std::memcpy(columns, s->matrix.columns.data(), s->matrix.columns.size() * 4);
  std::memcpy(values, s->matrix.values.data(), s->matrix.values.size() * 8);
}
void orc_study_free_numbering(const orc_study* s, uint32_t* out) {
  std::memcpy(out, s->free.data(), s->free.size() * 4);
}

// The hierarchy setup built, in f64, for comparison with the product's.
uint64_t orc_mg_levels(const orc_study* s) { return s->mg.levels.size(); }
void orc_mg_level_info(const orc_study* s, uint64_t level, orc_level_info* info) {
  const Level& lv = s->mg.levels[level];
  info->rows = lv.a.rows;
  info->row_block = lv.a.row_block;
  info->blocks = lv.a.columns.size();
  info->lambda_min = lv.lambda_min;
  info->lambda_max = lv.lambda_max;
  info->has_prolongator = lv.has_prolongator ? 1 : 0;
  info->p_blocks = lv.has_prolongator ? lv.prolongator.columns.size() : 0;
  info->p_col_block = lv.has_prolongator ? lv.prolongator.col_block : 0;
  info->has_factor = lv.has_factor ? 1 : 0;
}
void orc_mg_level_matrix(const orc_study* s, uint64_t level, int prolongator, uint64_t* starts,
                         uint32_t* columns, double* values) {
  const Level& lv = s->mg.levels[level];
  const BlockCsr<double>& m = prolongator ? lv.prolongator : lv.a;
  for (size_t i = 0; i <= m.rows; ++i) starts[i] = m.starts[i];
  std::memcpy(columns, m.columns.data(), m.columns.size() * 4);
  std::memcpy(values, m.values.data(), m.values.size() * 8);
}
void orc_mg_level_inverse_diagonal(const orc_study* s, uint64_t level, double* out) {
  const Level& lv = s->mg.levels[level];
  std::memcpy(out, lv.inverse_diagonal.data(), lv.inverse_diagonal.size() * 8);
}
void orc_mg_level_aggregates(const orc_study* s, uint64_t level, uint32_t* out) {
  const Level& lv = s->mg.levels[level];
  std::memcpy(out, lv.aggregates.data(), lv.aggregates.size() * 4);
}
void orc_mg_get_stats(const orc_study* s, orc_mg_stats* st) { s->mg.stats(st); }
// One V-cycle (or Jacobi application) in the study's precision: Preconditioner::apply.
void orc_precondition(orc_study* s, const double* r, double* z) { s->pcg.precondition(r, z); }
// The f64 system product, csr.rs:112-120.
void orc_system_multiply(orc_study* s, const double* x, double* y) { s->pcg.system_multiply(x, y); }
double orc_multiply_rounding_bound(const orc_study* s, const double* x) {
  return s->matrix.multiply_rounding_bound(x);
}

// ---------------------------------------------------------------------------------------------
// Stages of one level of the V-cycle in the study's precision, with the per-entry rounding bounds
// the reference's device tests assert against (crates/solidfem-solve/src/gpu/reference.rs:256-355;
// tests/solver/gpu_cycle_execution.rs:253-267): a device stage and this one each lie within the
// bound of the exact value of the same rounded inputs, so they differ by at most twice the bound.
// Inputs arrive in f64 and are rounded to the cycle's vector type; outputs are widened to f64.
// ---------------------------------------------------------------------------------------------
}  // extern "C"

namespace {

// |M| |v| for a block matrix, in f64.
template <class S>
vector<double> abs_product(const BlockCsr<S>& m, const vector<double>& v) {
  const size_t rb = m.row_block, cb = m.col_block;
  vector<double> out(m.rows * rb, 0.0);
  for (size_t row = 0; row < m.rows; ++row)
    for (size_t at = m.starts[row]; at < m.starts[row + 1]; ++at) {
      const S* b = m.block(at);
      const size_t col = (size_t)m.columns[at] * cb;
      for (size_t p = 0; p < rb; ++p)
        for (size_t q = 0; q < cb; ++q) out[row * rb + p] += std::fabs((double)b[p * cb + q]) * std::fabs(v[col + q]);
    }
  return out;
}

// reference.rs:256-274: terms * unit * sum |a_ij x_j| per scalar row.
template <class S>
vector<double> multiply_bound(const BlockCsr<S>& m, const vector<double>& x, double unit) {
  vector<double> out = abs_product(m, x);
  for (size_t row = 0; row < m.rows; ++row) {
    const double terms = (double)(m.starts[row + 1] - m.starts[row]) * (double)m.col_block;
    for (size_t p = 0; p < m.row_block; ++p) out[row * m.row_block + p] *= terms * unit;
  }
  return out;
}

// The transpose of a block matrix (the stored restriction), values widened to f64.
template <class S>
BlockCsr<double> transpose(const BlockCsr<S>& m, size_t out_rows) {
  BlockCsr<double> t;
  t.rows = out_rows;
  t.row_block = m.col_block;
  t.col_block = m.row_block;
  t.starts.assign(out_rows + 1, 0);
  for (uint32_t c : m.columns) t.starts[c + 1] += 1;
  for (size_t i = 0; i < out_rows; ++i) t.starts[i + 1] += t.starts[i];
  vector<size_t> at(t.starts.begin(), t.starts.end() - 1);
  t.columns.resize(m.columns.size());
  t.values.resize(m.values.size());
  const size_t rb = m.row_block, cb = m.col_block;
  for (size_t row = 0; row < m.rows; ++row)
    for (size_t k = m.starts[row]; k < m.starts[row + 1]; ++k) {
      const size_t slot = at[m.columns[k]]++;
      t.columns[slot] = (uint32_t)row;
      for (size_t p = 0; p < rb; ++p)
        for (size_t q = 0; q < cb; ++q) t.values[slot * rb * cb + q * rb + p] = (double)m.block(k)[p * cb + q];
    }
  return t;
}

// y = blockdiag(d) x, f64.
void block_apply(const vector<double>& d, size_t n, const vector<double>& x, vector<double>& y) {
  y.assign(x.size(), 0.0);
  for (size_t row = 0; row < x.size() / n; ++row)
    for (size_t p = 0; p < n; ++p) {
      double sum = 0.0;
      for (size_t q = 0; q < n; ++q) sum += d[(row * n + p) * n + q] * x[row * n + q];
      y[row * n + p] = sum;
    }
}

// reference.rs:276-355: a first-order bound on |computed - exact| of the smoother from zero on
// right-hand side b (already in the vector type), with the scalars rounded to that type; the
// division by theta allowed 2.5 units of rounding.
template <class S, class V>
vector<double> smoother_bound(const SLevel<S>& lv, size_t degree, const vector<double>& b, double unit) {
  const BlockCsr<S>& a = lv.a;
  const size_t n = a.row_block, len = a.rows * n;
  vector<double> diag(lv.inv.size()), abs_diag(lv.inv.size());
  for (size_t i = 0; i < diag.size(); ++i) {
    diag[i] = (double)lv.inv[i];
    abs_diag[i] = std::fabs(diag[i]);
  }
  const double theta0 = 0.5 * (lv.lambda_max + lv.lambda_min), delta = 0.5 * (lv.lambda_max - lv.lambda_min);
  const double sigma = theta0 / delta;
  double rho = 1.0 / sigma;
  const double theta = (double)(V)theta0;
  vector<double> abs_b(len), z, abs_bb, work, abs_work, propagated;
  for (size_t i = 0; i < len; ++i) abs_b[i] = std::fabs(b[i]);
  block_apply(abs_diag, n, abs_b, abs_bb);
  block_apply(diag, n, b, z);
  vector<double> residual(b), direction(len), solution(len), error_d(len), error_r(len, 0.0);
  for (size_t i = 0; i < len; ++i) {
    error_d[i] = ((double)n * unit * abs_bb[i]) / std::fabs(theta) + 2.5 * unit * std::fabs(z[i] / theta);
    direction[i] = z[i] / theta;
    solution[i] = direction[i];
  }
  vector<double> error_x(error_d), terms(len);
  for (size_t row = 0; row < a.rows; ++row)
    for (size_t p = 0; p < n; ++p) terms[row * n + p] = (double)(a.starts[row + 1] - a.starts[row]) * (double)a.col_block;
  vector<double> abs_direction(len), ad(len), abs_residual(len);
  for (size_t s = 1; s < degree; ++s) {
    const double next = 1.0 / (2.0 * sigma - rho);
    const double c1 = (double)(V)(next * rho), c2 = (double)(V)(2.0 * next / delta);
    rho = next;
    for (size_t i = 0; i < len; ++i) abs_direction[i] = std::fabs(direction[i]);
    abs_work = abs_product(a, abs_direction);
    propagated = abs_product(a, error_d);
    for (size_t row = 0; row < a.rows; ++row) {  // residual -= A direction, exact enough in f64
      double out[8];
      a.multiply_row(row, direction.data(), out);
      for (size_t p = 0; p < n; ++p) residual[row * n + p] -= out[p];
    }
    for (size_t i = 0; i < len; ++i)
      error_r[i] += terms[i] * unit * abs_work[i] + propagated[i] + unit * std::fabs(residual[i]);
    block_apply(diag, n, residual, z);
    for (size_t i = 0; i < len; ++i) abs_residual[i] = std::fabs(residual[i]);
    block_apply(abs_diag, n, abs_residual, abs_work);
    block_apply(abs_diag, n, error_r, work);
    for (size_t i = 0; i < len; ++i) {
      const double error_z = (double)n * unit * abs_work[i] + work[i];
      const double d = c1 * direction[i] + c2 * z[i];
      error_d[i] = std::fabs(c1) * error_d[i] + std::fabs(c2) * error_z +
                   3.0 * unit * (std::fabs(c1 * direction[i]) + std::fabs(c2 * z[i]));
      direction[i] = d;
      solution[i] += d;
      error_x[i] += error_d[i] + unit * std::fabs(solution[i]);
    }
  }
  return error_x;
}

template <class S, class V>
int level_stage(Cycle<S, V>& c, size_t li, int stage, const double* in0, const double* in1, double* out,
                double* bound) {
  if (li >= c.levels.size()) return 1;
  SLevel<S>& lv = c.levels[li];
  auto& w = c.work[li];
  const size_t n = lv.a.dofs(), rb = lv.a.row_block;
  const double unit = std::is_same<V, float>::value ? (double)FLT_EPSILON : DBL_EPSILON;
  auto rounded = [](const double* p, size_t len) {
    vector<V> v(len);
    for (size_t i = 0; i < len; ++i) v[i] = (V)p[i];
    return v;
  };
  auto widened = [](const vector<V>& v) { return vector<double>(v.begin(), v.end()); };
  switch (stage) {
    case ORC_STAGE_SMOOTH:
    case ORC_STAGE_SMOOTH_ADD: {
      if (lv.factor && !lv.has_p) return 1;
      vector<V> b = rounded(in0, n), x(n);
      c.smooth(li, b.data(), x.data());
      vector<double> e = smoother_bound<S, V>(lv, c.degree, widened(b), unit);
      if (stage == ORC_STAGE_SMOOTH_ADD) {
        vector<V> base = rounded(in1, n);
        for (size_t i = 0; i < n; ++i) {
          x[i] = base[i] + x[i];
          e[i] += unit * std::fabs((double)x[i]);
        }
      }
      for (size_t i = 0; i < n; ++i) {
        out[i] = (double)x[i];
        bound[i] = e[i];
      }
      return 0;
    }
    case ORC_STAGE_START: {  // cycle.rs:591-610: d = (D^-1 b) / theta, the smoother's first x
      vector<V> b = rounded(in0, n), z(n);
      const V first = (V)(0.5 * (lv.lambda_max + lv.lambda_min));
      vector<double> abs_b(n), abs_bb, zz;
      for (size_t row = 0; row < lv.a.rows; ++row) c.apply_inverse_diagonal(lv, row, b.data(), z.data());
      vector<double> diag(lv.inv.size());
      for (size_t i = 0; i < diag.size(); ++i) diag[i] = std::fabs((double)lv.inv[i]);
      for (size_t i = 0; i < n; ++i) abs_b[i] = std::fabs((double)b[i]);
      block_apply(diag, rb, abs_b, abs_bb);
      for (size_t i = 0; i < n; ++i) {
        const V d = z[i] / first;
        out[i] = (double)d;
        bound[i] = ((double)rb * unit * abs_bb[i]) / std::fabs((double)first) + 2.5 * unit * std::fabs((double)d);
      }
      return 0;
    }
    case ORC_STAGE_RESIDUAL: {  // cycle.rs:548-564; bound as gpu_cycle_execution.rs:253-267
      vector<V> b = rounded(in0, n), x = rounded(in1, n), r(n);
      c.residual(li, b.data(), x.data(), r.data());
      vector<double> xd = widened(x), e = multiply_bound(lv.a, xd, unit), ax = abs_product(lv.a, xd);
      for (size_t i = 0; i < n; ++i) {
        out[i] = (double)r[i];
        bound[i] = e[i] + unit * (std::fabs((double)b[i]) + ax[i]);
      }
      return 0;
    }
    case ORC_STAGE_RESTRICT: {  // block.rs:157-172 (the reference's device restricts by the stored transpose)
      if (!lv.has_p) return 1;
      const size_t cn = c.levels[li + 1].a.dofs();
      vector<V> r = rounded(in0, n), y(cn);
      lv.p.multiply_transpose(r.data(), y.data(), cn);
      BlockCsr<double> t = transpose(lv.p, c.levels[li + 1].a.rows);
      vector<double> e = multiply_bound(t, widened(r), unit);
      for (size_t i = 0; i < cn; ++i) {
        out[i] = (double)y[i];
        bound[i] = e[i];
      }
      return 0;
    }
    case ORC_STAGE_PROLONG: {  // cycle.rs:512-521: x += P e
      if (!lv.has_p) return 1;
      const size_t cn = c.levels[li + 1].a.dofs();
      vector<V> e = rounded(in0, cn), x = rounded(in1, n), pe(rb);
      vector<double> ed = widened(e), eb = multiply_bound(lv.p, ed, unit), ap = abs_product(lv.p, ed);
      for (size_t row = 0; row < lv.a.rows; ++row) {
        lv.p.multiply_row(row, e.data(), pe.data());
        for (size_t p = 0; p < rb; ++p) {
          const size_t i = row * rb + p;
          out[i] = (double)(V)(x[i] + pe[p]);
          bound[i] = eb[i] + unit * (std::fabs((double)x[i]) + ap[i]);
        }
      }
      return 0;
    }
  }
  (void)w;
  return 1;
}

}  // namespace

extern "C" {

int orc_level_stage(orc_study* s, uint64_t level, int stage, const double* in0, const double* in1, double* out,
                    double* bound) {
  if (!s->use_mg) return 1;
  switch (s->mg.precision) {
    case ORC_PRECISION_DOUBLE: return level_stage(s->mg.dd, level, stage, in0, in1, out, bound);
    case ORC_PRECISION_SINGLE_STORAGE: return level_stage(s->mg.fd, level, stage, in0, in1, out, bound);
    default: return level_stage(s->mg.ff, level, stage, in0, in1, out, bound);
  }
}

// StaticStudy::solution, study.rs:246-260: recovery of the current displacements.
int orc_study_recover(orc_study* s) {
  double t0 = now_seconds();
  vector<P3> disp(s->free.size());
  vector<double> flat(3 * s->free.size());
  orc_study_displacements(s, flat.data());
  for (size_t n = 0; n < disp.size(); ++n) disp[n] = {flat[3 * n], flat[3 * n + 1], flat[3 * n + 2]};
  int c = recover(s->mesh->q, s->field, s->quadrature, disp, s->recovered);
  s->seconds[3] += now_seconds() - t0;
  s->recovered_done = c == 0;
  return c;
}
// Recovery of caller-given displacements (every mesh node, x 3), for comparing recovery alone.
int orc_study_recover_with(orc_study* s, const double* flat) {
  vector<P3> disp(s->free.size());
  for (size_t n = 0; n < disp.size(); ++n) disp[n] = {flat[3 * n], flat[3 * n + 1], flat[3 * n + 2]};
  int c = recover(s->mesh->q, s->field, s->quadrature, disp, s->recovered);
  s->recovered_done = c == 0;
  return c;
}

void orc_study_nodal_stress(const orc_study* s, double* stress6, double* von_mises_out) {
  for (size_t n = 0; n < s->recovered.nodal_stress.size(); ++n) {
    for (int k = 0; k < 6; ++k) stress6[6 * n + k] = s->recovered.nodal_stress[n][k];
    von_mises_out[n] = s->recovered.nodal_von_mises[n];
  }
}
uint64_t orc_study_point_count(const orc_study* s) { return s->recovered.points.size(); }
void orc_study_point_stresses(const orc_study* s, orc_point_stress* out) {
  std::memcpy(out, s->recovered.points.data(), s->recovered.points.size() * sizeof(orc_point_stress));
}

// Element stiffness of one element (element.rs:98-133), for element-level tests.
int orc_element_stiffness(const double nodes[30], const orc_material* material, int quadrature,
                          double ke[900]) {
  P3 n[10];
  for (int a = 0; a < 10; ++a) n[a] = {nodes[3 * a], nodes[3 * a + 1], nodes[3 * a + 2]};
  MaterialField f;
  f.spec = *material;
  return element_stiffness(n, f, quadrature, ke);
}

}  // extern "C"
