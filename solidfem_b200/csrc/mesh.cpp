// Host-side mesh input: the structured box, the 10-node upgrade and the boundary faces. Node order
// decides the free numbering and therefore the multigrid aggregates, so the numbering follows the
// reference exactly: crates/solidfem-mesh/src/{box_mesh.rs,tet.rs,quadratic.rs,boundary.rs}.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <ctime>
#include <cstdio>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "sf_internal.h"

namespace sf {

const int kFaceNodes[4][6] = {{1, 2, 3, 5, 9, 8}, {0, 3, 2, 7, 9, 6}, {0, 1, 3, 4, 8, 7}, {0, 2, 1, 6, 5, 4}};
const int kEdgeCorners[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};

static thread_local sf_error g_error;

sf_error& error_slot() { return g_error; }

sf_status fail(sf_status status, const char* message) {
  g_error.status = status;
  std::snprintf(g_error.message, sizeof(g_error.message), "%s", message ? message : "");
  return status;
}

int default_threads() {
#ifdef _OPENMP
  int logical = omp_get_num_procs();
#else
  int logical = 1;
#endif
  return std::max(1, std::min(8, logical / 2));
}

double now_seconds() {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

namespace {

typedef array<uint32_t, 3> Key3;

Key3 face_key(const array<uint32_t, 4>& t, int face) {
  Key3 k = {t[kFaceNodes[face][0]], t[kFaceNodes[face][1]], t[kFaceNodes[face][2]]};
  std::sort(k.begin(), k.end());
  return k;
}

// Signed volume, crates/solidfem-mesh/src/tet.rs:9-16.
double tet_volume(const P3& a, const P3& b, const P3& c, const P3& d) {
  double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  double v[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  double w[3] = {d[0] - a[0], d[1] - a[1], d[2] - a[2]};
  double det = u[0] * (v[1] * w[2] - v[2] * w[1]) - u[1] * (v[0] * w[2] - v[2] * w[0]) +
               u[2] * (v[0] * w[1] - v[1] * w[0]);
  return det / 6.0;
}

// Determinant over the longest edge cubed, tet.rs:28-44.
double relative_volume(const P3& a, const P3& b, const P3& c, const P3& d, double volume) {
  auto ls = [](const P3& p, const P3& q) {
    return (p[0] - q[0]) * (p[0] - q[0]) + (p[1] - q[1]) * (p[1] - q[1]) + (p[2] - q[2]) * (p[2] - q[2]);
  };
  double longest = 0.0;
  for (double x : {ls(a, b), ls(a, c), ls(a, d), ls(b, c), ls(b, d), ls(c, d)}) longest = std::max(longest, x);
  return 6.0 * volume / (longest * std::sqrt(longest));
}

// TetMesh::new's refusals, tet.rs:59-109.
sf_status validate(const vector<P3>& pos, const vector<array<uint32_t, 4>>& tets) {
  if (tets.empty()) return fail(SF_MESH_EMPTY, "the mesh has no tetrahedra");
  for (size_t n = 0; n < pos.size(); ++n)
    for (double c : pos[n])
      if (!std::isfinite(c)) {
        error_slot().node = (uint32_t)n;
        return fail(SF_MESH_NON_FINITE_POSITION, "a node position is not finite");
      }
  vector<char> used(pos.size(), 0);
  for (size_t t = 0; t < tets.size(); ++t) {
    for (uint32_t n : tets[t]) {
      if (n >= pos.size()) {
        error_slot().tet = (uint32_t)t;
        error_slot().node = n;
        return fail(SF_MESH_NODE_OUT_OF_RANGE, "a tetrahedron names a node that does not exist");
      }
      used[n] = 1;
    }
    const auto& v = tets[t];
    double vol = tet_volume(pos[v[0]], pos[v[1]], pos[v[2]], pos[v[3]]);
    if (std::isnan(vol) || vol <= 0.0) {
      error_slot().tet = (uint32_t)t;
      error_slot().value = vol;
      return fail(SF_MESH_DEGENERATE_TET, "a tetrahedron has no positive volume");
    }
    double rel = relative_volume(pos[v[0]], pos[v[1]], pos[v[2]], pos[v[3]], vol);
    if (std::isnan(rel) || rel < 1e-12) {
      error_slot().tet = (uint32_t)t;
      error_slot().value = rel;
      return fail(SF_MESH_FLAT_TET, "a tetrahedron is flat to rounding");
    }
  }
  for (size_t n = 0; n < used.size(); ++n)
    if (!used[n]) {
      error_slot().node = (uint32_t)n;
      return fail(SF_MESH_UNUSED_NODE, "a node belongs to no tetrahedron");
    }
  vector<Key3> faces;
  faces.reserve(tets.size() * 4);
  for (auto& t : tets)
    for (int f = 0; f < 4; ++f) faces.push_back(face_key(t, f));
  std::sort(faces.begin(), faces.end());
  for (size_t i = 0; i + 2 < faces.size(); ++i)
    if (faces[i] == faces[i + 2]) return fail(SF_MESH_NON_MANIFOLD_FACE, "a face is shared by more than two tetrahedra");
  return SF_OK;
}

// QuadraticTetMesh::from_linear (quadratic.rs:24-71) and boundary_faces (quadratic.rs:89-124).
void upgrade(vector<P3>&& pos, vector<array<uint32_t, 4>>&& tets, Mesh& out) {
  out.vertex_count = pos.size();
  vector<uint64_t> edges(tets.size() * 6);
  for (size_t t = 0; t < tets.size(); ++t)
    for (int e = 0; e < 6; ++e) {
      uint32_t x = tets[t][kEdgeCorners[e][0]], y = tets[t][kEdgeCorners[e][1]];
      edges[6 * t + e] = ((uint64_t)std::min(x, y) << 32) | std::max(x, y);
    }
  std::sort(edges.begin(), edges.end());
  edges.erase(std::unique(edges.begin(), edges.end()), edges.end());
  out.nodes = std::move(pos);
  out.nodes.resize(out.vertex_count + edges.size());
  for (size_t i = 0; i < edges.size(); ++i) {
    const P3& p = out.nodes[edges[i] >> 32];
    const P3& q = out.nodes[edges[i] & 0xffffffffu];
    out.nodes[out.vertex_count + i] = {0.5 * (p[0] + q[0]), 0.5 * (p[1] + q[1]), 0.5 * (p[2] + q[2])};
  }
  out.tets.resize(tets.size());
  for (size_t t = 0; t < tets.size(); ++t) {
    for (int i = 0; i < 4; ++i) out.tets[t][i] = tets[t][i];
    for (int e = 0; e < 6; ++e) {
      uint32_t x = tets[t][kEdgeCorners[e][0]], y = tets[t][kEdgeCorners[e][1]];
      uint64_t key = ((uint64_t)std::min(x, y) << 32) | std::max(x, y);
      out.tets[t][4 + e] = (uint32_t)(out.vertex_count + (std::lower_bound(edges.begin(), edges.end(), key) - edges.begin()));
    }
  }
  out.corners = std::move(tets);
  // Boundary faces: keys (sorted corners, tet, face) sorted, unique keys kept.
  struct Keyed {
    Key3 key;
    uint32_t tet;
    uint32_t face;
    bool operator<(const Keyed& o) const {
      if (key != o.key) return key < o.key;
      if (tet != o.tet) return tet < o.tet;
      return face < o.face;
    }
  };
  vector<Keyed> keyed(out.corners.size() * 4);
  for (size_t t = 0; t < out.corners.size(); ++t)
    for (int f = 0; f < 4; ++f) keyed[4 * t + f] = {face_key(out.corners[t], f), (uint32_t)t, (uint32_t)f};
  std::sort(keyed.begin(), keyed.end());
  out.faces.clear();
  for (size_t at = 0; at < keyed.size();) {
    size_t end = at + 1;
    while (end < keyed.size() && keyed[end].key == keyed[at].key) ++end;
    if (end == at + 1) {
      sf_boundary_face bf;
      bf.tet = keyed[at].tet;
      bf.face = keyed[at].face;
      for (int s = 0; s < 6; ++s) bf.nodes[s] = out.tets[bf.tet][kFaceNodes[bf.face][s]];
      out.faces.push_back(bf);
    }
    at = end;
  }
}

}  // namespace

sf_status build_linear_mesh(const double* positions, uint64_t n, const uint32_t* tets, uint64_t ntets,
                            Mesh& out) {
  vector<P3> pos(n);
  for (uint64_t i = 0; i < n; ++i) pos[i] = {positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]};
  vector<array<uint32_t, 4>> t(ntets);
  for (uint64_t i = 0; i < ntets; ++i)
    for (int k = 0; k < 4; ++k) t[i][k] = tets[4 * i + k];
  if (sf_status s = validate(pos, t)) return s;
  upgrade(std::move(pos), std::move(t), out);
  return SF_OK;
}

// box_tet_mesh, crates/solidfem-mesh/src/box_mesh.rs:22-90.
sf_status build_box_mesh(const double origin[3], const double size[3], const uint64_t div[3], Mesh& out) {
  for (int a = 0; a < 3; ++a)
    if (div[a] == 0) return fail(SF_MESH_INVALID_BOX, "each axis needs at least one division");
  for (int a = 0; a < 3; ++a)
    if (std::isnan(size[a]) || size[a] <= 0.0) return fail(SF_MESH_INVALID_BOX, "each box length must be positive");
  size_t dims[3] = {div[0] + 1, div[1] + 1, div[2] + 1};
  auto coord = [](double o, double s, size_t i, size_t d) {
    return i == d ? o + s : o + s * ((double)i / (double)d);
  };
  vector<P3> pos;
  pos.reserve(dims[0] * dims[1] * dims[2]);
  for (size_t k = 0; k < dims[2]; ++k)
    for (size_t j = 0; j < dims[1]; ++j)
      for (size_t i = 0; i < dims[0]; ++i)
        pos.push_back({coord(origin[0], size[0], i, div[0]), coord(origin[1], size[1], j, div[1]),
                       coord(origin[2], size[2], k, div[2])});
  // Six tets per cell around the body diagonal: axis orders with their orientation.
  static const int kOrders[6][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}, {0, 2, 1}, {2, 1, 0}, {1, 0, 2}};
  vector<array<uint32_t, 4>> tets;
  tets.reserve(6 * div[0] * div[1] * div[2]);
  auto index = [&](const size_t at[3]) { return (uint32_t)(at[0] + dims[0] * (at[1] + dims[1] * at[2])); };
  for (size_t k = 0; k < div[2]; ++k)
    for (size_t j = 0; j < div[1]; ++j)
      for (size_t i = 0; i < div[0]; ++i)
        for (int o = 0; o < 6; ++o) {
          size_t at[3] = {i, j, k};
          uint32_t v[4];
          v[0] = index(at);
          for (int s = 0; s < 3; ++s) {
            at[kOrders[o][s]] += 1;
            v[s + 1] = index(at);
          }
          if (o < 3)
            tets.push_back({v[0], v[1], v[2], v[3]});
          else
            tets.push_back({v[0], v[2], v[1], v[3]});
        }
  if (sf_status s = validate(pos, tets)) return s;
  upgrade(std::move(pos), std::move(tets), out);
  return SF_OK;
}

// QuadraticTetMesh::face_connected_bodies, quadratic.rs:129-166.
vector<vector<uint32_t>> face_connected_bodies(const Mesh& mesh) {
  size_t n = mesh.tets.size();
  vector<size_t> parent(n);
  std::iota(parent.begin(), parent.end(), 0);
  auto find = [&](size_t x) {
    while (parent[x] != x) {
      parent[x] = parent[parent[x]];
      x = parent[x];
    }
    return x;
  };
  // Tets sharing a face are joined. Faces are bucketed by their smallest corner (a counting sort:
  // a shared face has the same sorted key in both tets, so both copies land in one bucket of a
  // few faces, and buckets follow node order, which keeps the passes cache-friendly); inside a
  // bucket, equal keys pair their tets. Keys, bucket counts and pairs are found in parallel, the
  // joins run in one thread. Joining makes the smallest tet of a body its root, so the partition
  // and the body order below (by first tet) do not depend on the order of the joins: they are the
  // ones a sort of the keys gives.
  const size_t nodes = mesh.nodes.size(), faces = 4 * n;
  int threads = 1;
#ifdef _OPENMP
  threads = n < 16384 ? 1 : std::max(1, std::min(omp_get_max_threads(), 16));
#endif
  vector<uint32_t> low(faces);
  vector<uint64_t> key(faces);  // the key's two larger corners
#ifdef _OPENMP
#pragma omp parallel for num_threads(threads) schedule(static)
#endif
  for (long long t = 0; t < (long long)n; ++t)
    for (int f = 0; f < 4; ++f) {
      Key3 k = face_key(mesh.corners[t], f);
      low[4 * t + f] = k[0];
      key[4 * t + f] = ((uint64_t)k[1] << 32) | k[2];
    }
  // per-thread counts over contiguous face ranges, then each thread's place inside every bucket
  vector<vector<uint32_t>> counts(threads, vector<uint32_t>(nodes + 1, 0));
#ifdef _OPENMP
#pragma omp parallel for num_threads(threads) schedule(static, 1)
#endif
  for (int c = 0; c < threads; ++c) {
    const size_t b0 = faces * c / threads, b1 = faces * (c + 1) / threads;
    for (size_t i = b0; i < b1; ++i) counts[c][low[i]] += 1;
  }
  vector<uint32_t> start(nodes + 1, 0);
  for (size_t v = 0; v < nodes; ++v) {
    uint32_t at = start[v];
    for (int c = 0; c < threads; ++c) {
      const uint32_t k = counts[c][v];
      counts[c][v] = at;
      at += k;
    }
    start[v + 1] = at;
  }
  vector<uint32_t> item(faces);
  vector<uint64_t> rest(faces);
#ifdef _OPENMP
#pragma omp parallel for num_threads(threads) schedule(static, 1)
#endif
  for (int c = 0; c < threads; ++c) {
    const size_t b0 = faces * c / threads, b1 = faces * (c + 1) / threads;
    for (size_t i = b0; i < b1; ++i) {
      const uint32_t at = counts[c][low[i]]++;
      item[at] = (uint32_t)(i / 4);
      rest[at] = key[i];
    }
  }
  vector<vector<std::pair<uint32_t, uint32_t>>> pairs(threads);
#ifdef _OPENMP
#pragma omp parallel for num_threads(threads) schedule(static, 1)
#endif
  for (int c = 0; c < threads; ++c) {
    const size_t v0 = nodes * c / threads, v1 = nodes * (c + 1) / threads;
    for (size_t v = v0; v < v1; ++v)
      for (uint32_t i = start[v]; i < start[v + 1]; ++i)
        for (uint32_t j = i + 1; j < start[v + 1]; ++j)
          if (rest[i] == rest[j]) pairs[c].push_back({item[i], item[j]});
  }
  for (auto& list : pairs)
    for (auto& pr : list) {
      size_t a = find(pr.first), b = find(pr.second);
      if (a != b) parent[std::max(a, b)] = std::min(a, b);
    }
  vector<vector<uint32_t>> groups;
  vector<size_t> group_of(n, SIZE_MAX);
  for (size_t t = 0; t < n; ++t) {
    size_t r = find(t);
    if (group_of[r] == SIZE_MAX) {
      group_of[r] = groups.size();
      groups.emplace_back();
    }
    groups[group_of[r]].push_back((uint32_t)t);
  }
  return groups;
}

}  // namespace sf
