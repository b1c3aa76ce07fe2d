// The study state machine and the C ABI: Model -> StudyBuilder -> StaticStudy
// (crates/solidfem-elastic/src/study.rs), with the stiffness assembled on the device, the
// multigrid hierarchy built by the host setup (setup.cpp) and uploaded, and the conjugate gradient
// and V-cycle running on the device (solve.cu).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <future>
#include <map>
#include <numeric>
#include <memory>

#ifdef _OPENMP
#include <cuda.h>
#include <omp.h>
#endif

#include "device.h"
#include "sf_internal.h"
#include "batch.h"

using namespace sf;

struct sf_mesh {
  Mesh mesh;
};

struct sf_model {
  Model model;
};

namespace {

const double ON_BOUNDARY_EPS = 0;  // unused; faces are matched exactly

// Constraint check (crates/solidfem-elastic/src/constraints.rs:40-135): each face-connected body
// needs three non-collinear held nodes, a body held through a shared node counting as held.
double distance3(const P3& a, const P3& b) {
  double d[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
  return std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
}

int remaining_freedom(const vector<P3>& pts, double size) {  // 0 held, 1 free, 2 point, 3 line
  if (pts.empty()) return 1;
  double limit = 1e-9 * size;
  P3 first = pts[0], far = first;
  double fd = 0.0;
  for (auto& p : pts) {
    double d = distance3(first, p);
    if (d > fd) {
      far = p;
      fd = d;
    }
  }
  if (fd <= limit) return 2;
  double ax[3] = {(far[0] - first[0]) / fd, (far[1] - first[1]) / fd, (far[2] - first[2]) / fd};
  for (auto& p : pts) {
    double v[3] = {p[0] - first[0], p[1] - first[1], p[2] - first[2]};
    double along = v[0] * ax[0] + v[1] * ax[1] + v[2] * ax[2];
    double off[3] = {v[0] - along * ax[0], v[1] - along * ax[1], v[2] - along * ax[2]};
    if (std::sqrt(off[0] * off[0] + off[1] * off[1] + off[2] * off[2]) > limit) return 0;
  }
  return 3;
}

sf_status check_constraints(const Mesh& m, const vector<char>& fixed) {
  bool any = false;
  for (char f : fixed) any = any || f;
  if (!any) return fail(SF_NO_FIXED_NODES, "no node is fixed: the model is free to move");
  auto bodies = face_connected_bodies(m);
  vector<vector<uint32_t>> body_nodes(bodies.size());
  vector<double> sizes(bodies.size());
  vector<uint32_t> mark(m.nodes.size(), 0xffffffffu);
  for (size_t b = 0; b < bodies.size(); ++b) {
    // The body's nodes, ascending: every node when the mesh is one body (a valid mesh uses every
    // node), otherwise its tets' nodes deduplicated and sorted.
    vector<uint32_t>& nodes = body_nodes[b];
    if (bodies.size() == 1) {
      nodes.resize(m.nodes.size());
      std::iota(nodes.begin(), nodes.end(), 0u);
    } else {
      for (uint32_t t : bodies[b])
        for (uint32_t n : m.tets[t])
          if (mark[n] != (uint32_t)b) {
            mark[n] = (uint32_t)b;
            nodes.push_back(n);
          }
      std::sort(nodes.begin(), nodes.end());
    }
    P3 lo = {INFINITY, INFINITY, INFINITY}, hi = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t n : nodes)
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::min(lo[a], m.nodes[n][a]);
        hi[a] = std::max(hi[a], m.nodes[n][a]);
      }
    sizes[b] = distance3(lo, hi);
  }
  vector<char> held = fixed, anchored(bodies.size(), 0);
  for (bool changed = true; changed;) {
    changed = false;
    for (size_t b = 0; b < bodies.size(); ++b) {
      if (anchored[b]) continue;
      vector<P3> pts;
      for (uint32_t n : body_nodes[b])
        if (held[n]) pts.push_back(m.nodes[n]);
      if (remaining_freedom(pts, sizes[b]) == 0) {
        anchored[b] = 1;
        changed = true;
        for (uint32_t n : body_nodes[b]) held[n] = 1;
      }
    }
  }
  for (size_t b = 0; b < bodies.size(); ++b)
    if (!anchored[b]) {
      size_t count = 0;
      for (uint32_t n : body_nodes[b]) count += held[n] ? 1 : 0;
      error_slot().tet = bodies[b][0];
      error_slot().node = (uint32_t)count;
      return fail(SF_BODY_NOT_HELD, "a body is not held by three non-collinear nodes");
    }
  return SF_OK;
}

// check_held_dofs with its pivoted rank (constraints.rs:162-256).
sf_status check_held_dofs(const Mesh& m, const vector<char>& fixed,
                          const vector<std::pair<std::pair<uint32_t, uint32_t>, double>>& prescribed) {
  for (auto& body : face_connected_bodies(m)) {
    vector<char> in_body(m.nodes.size(), 0);
    vector<uint32_t> nodes;
    for (uint32_t t : body)
      for (uint32_t n : m.tets[t])
        if (!in_body[n]) {
          in_body[n] = 1;
          nodes.push_back(n);
        }
    std::sort(nodes.begin(), nodes.end());
    P3 lo = {INFINITY, INFINITY, INFINITY}, hi = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t n : nodes)
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::min(lo[a], m.nodes[n][a]);
        hi[a] = std::max(hi[a], m.nodes[n][a]);
      }
    double size = std::max(distance3(lo, hi), 2.2250738585072014e-308);
    double c[3] = {0, 0, 0};
    for (uint32_t n : nodes)
      for (int a = 0; a < 3; ++a) c[a] += m.nodes[n][a];
    for (int a = 0; a < 3; ++a) c[a] /= (double)nodes.size();
    vector<array<double, 6>> rows;
    auto add = [&](uint32_t node, uint32_t axis) {
      const P3& p = m.nodes[node];
      double x = (p[0] - c[0]) / size, y = (p[1] - c[1]) / size, z = (p[2] - c[2]) / size;
      if (axis == 0) rows.push_back({1, 0, 0, 0, z, -y});
      else if (axis == 1) rows.push_back({0, 1, 0, -z, 0, x});
      else rows.push_back({0, 0, 1, y, -x, 0});
    };
    for (uint32_t n : nodes)
      if (fixed[n])
        for (uint32_t a = 0; a < 3; ++a) add(n, a);
    for (auto& pr : prescribed) {
      uint32_t node = pr.first.first, axis = pr.first.second;
      if (node < m.nodes.size() && in_body[node] && axis < 3) add(node, axis);
    }
    size_t rank = 0;
    for (int col = 0; col < 6; ++col) {
      if (rank >= rows.size()) break;
      size_t best = rank;
      for (size_t r = rank + 1; r < rows.size(); ++r) {
        double a = std::fabs(rows[r][col]), b = std::fabs(rows[best][col]);
        if (a > b) best = r;  // ties keep the lower index, as max_by with then(b.cmp(a))
      }
      if (std::fabs(rows[best][col]) <= 1e-9) continue;
      std::swap(rows[rank], rows[best]);
      auto pivot = rows[rank];
      for (size_t r = rank + 1; r < rows.size(); ++r) {
        double f = rows[r][col] / pivot[col];
        if (f != 0.0)
          for (int k = col; k < 6; ++k) rows[r][k] -= f * pivot[k];
      }
      ++rank;
    }
    if (rank < 6) {
      error_slot().tet = body[0];
      error_slot().rank = rank;
      return fail(SF_DOFS_DO_NOT_HOLD, "the held components do not remove every rigid motion of a body");
    }
  }
  return SF_OK;
}

// Consistent traction load (crates/solidfem-elastic/src/loads.rs:10-41), 6-point triangle rule.
void add_traction(const Mesh& m, const sf_boundary_face& f, const double t[3], vector<double>& load) {
  static const double TA = 0.091576213509771, TB = 0.445948490915965;
  static const double WA = 0.109951743655322, WB = 0.223381589678011;
  const double pts[6][3] = {{TA, TA, WA}, {1.0 - 2.0 * TA, TA, WA}, {TA, 1.0 - 2.0 * TA, WA},
                            {TB, TB, WB}, {1.0 - 2.0 * TB, TB, WB}, {TB, 1.0 - 2.0 * TB, WB}};
  P3 pos[6];
  for (int i = 0; i < 6; ++i) pos[i] = m.nodes[f.nodes[i]];
  for (int q = 0; q < 6; ++q) {
    double r = pts[q][0], s = pts[q][1], w = pts[q][2];
    double l1 = 1.0 - r - s;
    double v[6] = {l1 * (2.0 * l1 - 1.0), r * (2.0 * r - 1.0), s * (2.0 * s - 1.0), 4.0 * l1 * r, 4.0 * r * s, 4.0 * s * l1};
    double dr[6] = {-(4.0 * l1 - 1.0), 4.0 * r - 1.0, 0.0, 4.0 * (l1 - r), 4.0 * s, -4.0 * s};
    double ds[6] = {-(4.0 * l1 - 1.0), 0.0, 4.0 * s - 1.0, -4.0 * r, 4.0 * r, 4.0 * (l1 - s)};
    double tr[3] = {0, 0, 0}, ts[3] = {0, 0, 0};
    for (int n = 0; n < 6; ++n)
      for (int a = 0; a < 3; ++a) {
        tr[a] += dr[n] * pos[n][a];
        ts[a] += ds[n] * pos[n][a];
      }
    double nm[3] = {tr[1] * ts[2] - tr[2] * ts[1], tr[2] * ts[0] - tr[0] * ts[2], tr[0] * ts[1] - tr[1] * ts[0]};
    double length = std::sqrt(nm[0] * nm[0] + nm[1] * nm[1] + nm[2] * nm[2]);
    double measure = 0.5 * length * w;
    for (int n = 0; n < 6; ++n)
      for (int a = 0; a < 3; ++a) load[3 * (size_t)f.nodes[n] + a] += t[a] * v[n] * measure;
  }
}

// The frame of the free nodes' rigid-body modes (free_rigid_body_modes, rigid_modes.rs:36-83): the
// centroid of the free nodes (summed in node order) and 1 / the largest offset from it. The modes
// themselves are made on the device from it (setup_rigid_modes).
void rigid_frame(const vector<P3>& nodes, const vector<uint32_t>& free, size_t free_count, double center[3],
                 double* scale) {
  double c[3] = {0, 0, 0};
  for (size_t n = 0; n < nodes.size(); ++n)
    if (free[n] != FIXED)
      for (int a = 0; a < 3; ++a) c[a] += nodes[n][a];
  double div = (double)std::max<size_t>(free_count, 1);
  for (int a = 0; a < 3; ++a) c[a] /= div;
  double reach = 0.0;
  for (size_t n = 0; n < nodes.size(); ++n)
    if (free[n] != FIXED)
      for (int a = 0; a < 3; ++a) reach = std::max(reach, std::fabs(nodes[n][a] - c[a]));
  for (int a = 0; a < 3; ++a) center[a] = c[a];
  *scale = reach > 0.0 ? 1.0 / reach : 1.0;
}

// An allocator whose resize leaves new elements uninitialised: the pattern's large arrays are
// written in full by the parallel pass that fills them, so a zero fill first (single-threaded,
// and the page faults of tens of MB with it) is pure cost.
// build_load (study.rs:696-735): nodal forces and consistent tractions into `load` (3 per node),
// refusing a node that does not exist, a non-finite value and a face off the boundary.
sf_status build_load(const Mesh& mesh, const Model& md, vector<double>& load) {
  const size_t nn = mesh.nodes.size();
  for (auto& f : md.forces) {
    if (f.first >= nn) {
      error_slot().node = f.first;
      return fail(SF_NODE_OUT_OF_RANGE, "a loaded node does not exist");
    }
    for (double c : f.second)
      if (!std::isfinite(c)) return fail(SF_NON_FINITE_LOAD, "a nodal force is not finite");
    for (int a = 0; a < 3; ++a) load[3 * (size_t)f.first + a] += f.second[a];
  }
  if (!md.tractions.empty()) {
    // A boundary face is fixed by its (tet, face): a per-tet mask of boundary faces, and the
    // face's nodes compared with the mesh's own entry, decide membership in the boundary list.
    vector<unsigned char> boundary_mask(mesh.tets.size(), 0);
    vector<uint32_t> entry(mesh.tets.size() * 4, 0);
    for (size_t i = 0; i < mesh.faces.size(); ++i) {
      const sf_boundary_face& f = mesh.faces[i];
      boundary_mask[f.tet] |= (unsigned char)(1u << f.face);
      entry[(size_t)f.tet * 4 + f.face] = (uint32_t)i;
    }
    auto on_boundary = [&](const sf_boundary_face& f) {
      if (f.tet >= mesh.tets.size() || f.face >= 4 || !(boundary_mask[f.tet] & (1u << f.face))) return false;
      const sf_boundary_face& g = mesh.faces[entry[(size_t)f.tet * 4 + f.face]];
      for (int i = 0; i < 6; ++i)
        if (g.nodes[i] != f.nodes[i]) return false;
      return true;
    };
    for (auto& tr : md.tractions) {
      if (!on_boundary(tr.first)) {
        error_slot().tet = tr.first.tet;
        error_slot().face = tr.first.face;
        return fail(SF_FACE_NOT_ON_BOUNDARY, "a traction face is not on the mesh boundary");
      }
      for (double c : tr.second)
        if (!std::isfinite(c)) return fail(SF_NON_FINITE_LOAD, "a traction is not finite");
      if (!mesh.dev) add_traction(mesh, tr.first, tr.second.data(), load);
    }
    // a mesh generated on a device: the same sums, made there from its node array
    if (mesh.dev) return device_traction_load(mesh, md.tractions, load);
  }
  return SF_OK;
}

template <typename T>
struct NoInit : std::allocator<T> {
  template <typename U>
  struct rebind {
    typedef NoInit<U> other;
  };
  NoInit() = default;
  template <typename U>
  NoInit(const NoInit<U>&) {}
  template <typename U>
  void construct(U* p) noexcept {
    ::new (static_cast<void*>(p)) U;
  }
  template <typename U, typename... A>
  void construct(U* p, A&&... a) {
    ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
  }
};
typedef vector<uint32_t, NoInit<uint32_t>> RawU32;

struct HostPattern {
  vector<uint32_t> starts;                 // block rows over free nodes
  RawU32 cols;
  // Node-to-element incidence (each node's elements ascending) and each free row's node: the
  // device gather walks them, so no per-block list of contributions is built on the host.
  vector<uint32_t> inc_start, inc, row_node;
};

// The free-node block pattern (assembly.rs:55-81, csr.rs:19-71), built row-parallel from
// node-to-element incidence, which is kept for the device assembly.
bool build_pattern(const Mesh& m, const vector<uint32_t>& free, size_t free_count, int threads, HostPattern& hp) {
  size_t nn = m.nodes.size(), ne = m.tets.size();
  vector<uint32_t>& inc_start = hp.inc_start;
  inc_start.assign(nn + 1, 0);
  for (auto& t : m.tets)
    for (uint32_t n : t) inc_start[n + 1] += 1;
  for (size_t i = 0; i < nn; ++i) inc_start[i + 1] += inc_start[i];
  vector<uint32_t> fill(inc_start.begin(), inc_start.end() - 1);
  vector<uint32_t>& inc = hp.inc;
  inc.resize(inc_start[nn]);
  for (size_t e = 0; e < ne; ++e)
    for (uint32_t n : m.tets[e]) inc[fill[n]++] = (uint32_t)e;
  vector<uint32_t>& row_node = hp.row_node;
  row_node.resize(free_count);
  for (size_t n = 0; n < nn; ++n)
    if (free[n] != FIXED) row_node[free[n]] = (uint32_t)n;
  // Per row its distinct columns (a per-thread marker array stamped with the row), then the
  // sorted columns.
  vector<uint32_t> counts(free_count, 0);
#ifdef _OPENMP
#pragma omp parallel num_threads(threads)
#endif
  {
    vector<uint32_t> mark(free_count, 0xffffffffu);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1024)
#endif
    for (long long r = 0; r < (long long)free_count; ++r) {
      uint32_t node = row_node[r], distinct = 0;
      for (uint32_t k = inc_start[node]; k < inc_start[node + 1]; ++k)
        for (uint32_t n : m.tets[inc[k]]) {
          uint32_t fc = free[n];
          if (fc != FIXED && mark[fc] != (uint32_t)r) {
            mark[fc] = (uint32_t)r;
            ++distinct;
          }
        }
      counts[r] = distinct;
    }
  }
  hp.starts.assign(free_count + 1, 0);
  for (size_t r = 0; r < free_count; ++r) hp.starts[r + 1] = hp.starts[r] + counts[r];
  hp.cols.resize(hp.starts[free_count]);
#ifdef _OPENMP
#pragma omp parallel num_threads(threads)
#endif
  {
    vector<uint32_t> mark(free_count, 0xffffffffu), cols;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1024)
#endif
    for (long long r = 0; r < (long long)free_count; ++r) {
      uint32_t node = row_node[r];
      cols.clear();
      for (uint32_t k = inc_start[node]; k < inc_start[node + 1]; ++k)
        for (uint32_t n : m.tets[inc[k]]) {
          uint32_t fc = free[n];
          if (fc != FIXED && mark[fc] != (uint32_t)r) {
            mark[fc] = (uint32_t)r;
            cols.push_back(fc);
          }
        }
      std::sort(cols.begin(), cols.end());
      std::copy(cols.begin(), cols.end(), hp.cols.begin() + hp.starts[r]);
    }
  }
  return true;
}

}  // namespace

struct sf_builder {
  Model model;
  sf_study_options options;
  vector<uint32_t> free;
  size_t free_count = 0;
  vector<double> rhs;
  vector<std::pair<size_t, double>> prescribed;  // (free dof, value), sorted
  size_t next = 0;
  bool prescribed_applied = false;
  HostPattern pattern;
  AssemblyDevice asmdev;
  DeviceSolver solver;
  SetupMachine* setup = nullptr;
  bool setup_finished = false;
  double* modes = nullptr;  // the finest level's near-null modes on the device, until the setup takes them
  double assembly_seconds = 0, preconditioner_seconds = 0;
  float assembly_ms = 0, setup_ms = 0;
  sf_status failure = SF_OK;
  int threads = 1;
  ~sf_builder() {
    if (setup) setup_destroy(setup);
  }
};

struct sf_study {
  Model model;
  sf_study_options options;
  vector<uint32_t> free;
  size_t free_count = 0;
  vector<double> rhs;
  vector<std::pair<size_t, double>> prescribed;
  HostPattern pattern;
  AssemblyDevice asmdev;
  DeviceSolver solver;
  vector<HostLevel> levels;
  sf_report report;
  int status = ST_ACTIVE;
  bool cancelled = false;
  PcgState last;
  double step_ms = 0;
  double assembly_ms = 0;
  PcgState* pinned = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  RecoveryDevice rec;              // the incidence tables every recovery of this study reads
  sf_recovery* answer = nullptr;   // the finished recovery of the converged displacements
  vector<sf_recovery*> recoveries; // every live recovery of this study, `answer` included
  void release_answer();
  void orphan_recoveries();
  ~sf_study() {
    release_answer();
    orphan_recoveries();
    pinned_release(pinned);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    dev_free_all(solver);
    if (solver.mesh_keep && solver.stream) cudaStreamSynchronize(solver.stream);
    solver.mesh_keep.reset();
    if (solver.stream) cudaStreamDestroy(solver.stream);
  }
};

// A resumable stress recovery of one snapshot of a study's displacements (Recovery,
// results.rs:97-124): its own device buffers, the study's incidence tables, and how far it got
// (elements first, then one patch fit per vertex).
struct sf_recovery {
  sf_study* study = nullptr;
  RecoveryDevice dev;
  uint64_t next_element = 0, next_vertex = 0;
  bool converged = false;  // a snapshot of the converged answer, not a preview
  vector<void*> owned;     // dev's own buffers
};

extern "C" {
static void recovery_free(sf_recovery* r);  // defined with the recovery entry points
}

void sf_study::release_answer() {
  if (answer) recovery_free(answer);
  answer = nullptr;
}

// The study goes first: its recoveries keep their handles (which the caller still destroys) but
// lose their device memory, which goes with the study's own.
void sf_study::orphan_recoveries() {
  for (sf_recovery* r : recoveries) {
    r->study = nullptr;
    r->owned.clear();
  }
  recoveries.clear();
}

// Frees a device-built pattern that no solver took over, on a stream of its own (no device-wide wait).
static void release_pattern(int device, DevicePattern& dp) {
  if (dp.allocations.empty()) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  cudaStream_t st = nullptr;
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  for (auto& al : dp.allocations) cudaFreeAsync(al.first, st);
  cudaStreamDestroy(st);
  dp.allocations.clear();
  cudaSetDevice(prev);
}

static void release_builder_device(sf_builder* b) {
  dev_free_all(b->solver);
  // the device-to-device copies from a generated mesh end before its arrays can be let go
  if (b->solver.mesh_keep && b->solver.stream) cudaStreamSynchronize(b->solver.stream);
  b->solver.mesh_keep.reset();
  if (b->solver.stream) cudaStreamDestroy(b->solver.stream);
  b->solver.stream = nullptr;
}

extern "C" {

sf_status sf_last_error(sf_error* out) {
  if (out) *out = error_slot();
  return (sf_status)error_slot().status;
}

int32_t sf_abi_version(void) { return SF_ABI_VERSION; }

const char* sf_status_message(sf_status s) {
  switch (s) {
    case SF_OK: return "ok";
    case SF_MESH_EMPTY: return "the mesh has no tetrahedra";
    case SF_MESH_NON_FINITE_POSITION: return "a node position is not finite";
    case SF_MESH_NODE_OUT_OF_RANGE: return "a tetrahedron names a node that does not exist";
    case SF_MESH_DEGENERATE_TET: return "a tetrahedron has no positive volume";
    case SF_MESH_FLAT_TET: return "a tetrahedron is flat to rounding";
    case SF_MESH_UNUSED_NODE: return "a node belongs to no tetrahedron";
    case SF_MESH_NON_MANIFOLD_FACE: return "a face is shared by more than two tetrahedra";
    case SF_MESH_INVALID_BOX: return "the box needs positive lengths and divisions";
    case SF_NO_FIXED_NODES: return "no node is fixed";
    case SF_BODY_NOT_HELD: return "a body is not held";
    case SF_NODE_OUT_OF_RANGE: return "a node index is out of range";
    case SF_NON_FINITE_LOAD: return "a load is not finite";
    case SF_FACE_NOT_ON_BOUNDARY: return "a traction face is not on the boundary";
    case SF_NO_EFFECTIVE_LOAD: return "the model has no effective load";
    case SF_ELEMENT_INVERTED_JACOBIAN: return "an element has an inverted integration point";
    case SF_ELEMENT_INVALID_MATERIAL: return "an integration point has an invalid material";
    case SF_JACOBI_DIAGONAL: return "a diagonal entry is not positive";
    case SF_CANCELLED: return "cancelled";
    case SF_NOT_FINISHED: return "not finished";
    case SF_AXIS_OUT_OF_RANGE: return "an axis is out of range";
    case SF_PRESCRIBED_ON_FIXED_NODE: return "a prescribed component is on a fixed node";
    case SF_DOFS_DO_NOT_HOLD: return "the held components do not hold a body";
    case SF_MG_BLOCK_STRUCTURE: return "the matrix does not group into 3x3 blocks";
    case SF_MG_NEAR_NULL_LENGTH: return "the near-null space has the wrong length";
    case SF_MG_NOT_POSITIVE_DEFINITE: return "a multigrid block is not positive definite";
    case SF_MG_POSITION_LENGTH: return "the block positions have the wrong length";
    case SF_MG_COARSEST_NOT_FACTORED: return "the coarsest level is not factored";
    case SF_MG_COARSE_LENGTH: return "the coarse vector has the wrong length";
    case SF_PCG_NOT_POSITIVE_DEFINITE: return "the system is not positive definite";
    case SF_PCG_NOT_CONVERGED: return "the solver did not converge";
    case SF_INVALID_ARGUMENT: return "invalid argument";
    case SF_CUDA_ERROR: return "CUDA error";
    case SF_DEVICE_MEMORY_BUDGET: return "the device memory budget is exceeded";
    case SF_NO_DEVICE: return "no CUDA device";
    case SF_DEVICE_WAIT_TIMEOUT: return "a device wait timed out";
  }
  return "unknown status";
}

// ------------------------------------------------------------------------------ mesh
sf_status sf_box_tet_mesh(const double origin[3], const double size[3], const uint64_t divisions[3], sf_mesh** out) {
  if (!origin || !size || !divisions || !out) return fail(SF_INVALID_ARGUMENT, "null argument");
  std::unique_ptr<sf_mesh> m(new sf_mesh);
  if (sf_status s = build_box_mesh(origin, size, divisions, m->mesh)) return s;
  *out = m.release();
  return SF_OK;
}

sf_status sf_mesh_from_linear(const double* positions, uint64_t n, const uint32_t* tets, uint64_t ntets, sf_mesh** out) {
  if ((!positions && n) || (!tets && ntets) || !out) return fail(SF_INVALID_ARGUMENT, "null argument");
  std::unique_ptr<sf_mesh> m(new sf_mesh);
  if (sf_status s = build_linear_mesh(positions, n, tets, ntets, m->mesh)) return s;
  *out = m.release();
  return SF_OK;
}

sf_status sf_box_tet_mesh_device(const double origin[3], const double size[3], const uint64_t divisions[3],
                                 int32_t device, sf_mesh** out) {
  if (!origin || !size || !divisions || !out) return fail(SF_INVALID_ARGUMENT, "null argument");
  std::unique_ptr<sf_mesh> m(new sf_mesh);
  if (sf_status s = build_box_mesh_device(origin, size, divisions, device, m->mesh)) return s;
  *out = m.release();
  return SF_OK;
}

sf_status sf_mesh_from_linear_device(const double* positions, uint64_t n, const uint32_t* tets, uint64_t ntets,
                                     int32_t device, sf_mesh** out) {
  if ((!positions && n) || (!tets && ntets) || !out) return fail(SF_INVALID_ARGUMENT, "null argument");
  std::unique_ptr<sf_mesh> m(new sf_mesh);
  if (sf_status s = build_linear_mesh_device(positions, n, tets, ntets, device, m->mesh)) return s;
  *out = m.release();
  return SF_OK;
}

sf_status sf_part_tet_mesh_device(const double* x_lines, uint64_t x_count, const double* y_lines, uint64_t y_count,
                                  const double* z_lines, uint64_t z_count, uint64_t wall_cells, int32_t device,
                                  sf_mesh** out) {
  if (!x_lines || !y_lines || !z_lines || !out) return fail(SF_INVALID_ARGUMENT, "null argument");
  const double* lines[3] = {x_lines, y_lines, z_lines};
  const uint64_t counts[3] = {x_count, y_count, z_count};
  for (int a = 0; a < 3; ++a)
    for (uint64_t i = 0; i < counts[a]; ++i)
      if (!std::isfinite(lines[a][i]) || (i > 0 && !(lines[a][i] > lines[a][i - 1])))
        return fail(SF_MESH_INVALID_BOX, "grid lines must be finite and strictly ascending");
  std::unique_ptr<sf_mesh> m(new sf_mesh);
  if (sf_status s = build_part_mesh_device(lines, counts, wall_cells, device, m->mesh)) return s;
  *out = m.release();
  return SF_OK;
}

int32_t sf_mesh_device(const sf_mesh* m) { return m && m->mesh.dev ? m->mesh.dev->device : -1; }

void sf_mesh_destroy(sf_mesh* m) { delete m; }
uint64_t sf_mesh_node_count(const sf_mesh* m) { return m ? m->mesh.nodes.size() : 0; }
uint64_t sf_mesh_tet_count(const sf_mesh* m) { return m ? m->mesh.tets.size() : 0; }
uint64_t sf_mesh_vertex_count(const sf_mesh* m) { return m ? m->mesh.vertex_count : 0; }
uint64_t sf_mesh_boundary_face_count(const sf_mesh* m) { return m ? m->mesh.faces.size() : 0; }

sf_status sf_mesh_nodes(const sf_mesh* m, double* out) {
  if (!m || !out) return fail(SF_INVALID_ARGUMENT, "null argument");
  std::memcpy(out, m->mesh.nodes.data(), m->mesh.nodes.size() * 24);
  return SF_OK;
}

sf_status sf_mesh_tets(const sf_mesh* m, uint32_t* out) {
  if (!m || !out) return fail(SF_INVALID_ARGUMENT, "null argument");
  std::memcpy(out, m->mesh.tets.data(), m->mesh.tets.size() * 40);
  return SF_OK;
}

sf_status sf_mesh_boundary_faces(const sf_mesh* m, sf_boundary_face* out) {
  if (!m || !out) return fail(SF_INVALID_ARGUMENT, "null argument");
  std::memcpy(out, m->mesh.faces.data(), m->mesh.faces.size() * sizeof(sf_boundary_face));
  return SF_OK;
}

// ------------------------------------------------------------------------------ model
sf_status sf_model_create(const sf_mesh* mesh, sf_material material, sf_model** out) {
  if (!mesh || !out) return fail(SF_INVALID_ARGUMENT, "null argument");
  sf_model* m = new sf_model;
  m->model.mesh = mesh->mesh;
  m->model.material.kind = MATERIAL_UNIFORM;
  m->model.material.uniform = material;
  *out = m;
  return SF_OK;
}

void sf_model_destroy(sf_model* m) { delete m; }

sf_status sf_model_set_material_field(sf_model* m, sf_material_field_fn field, void* user) {
  if (!m || !field) return fail(SF_INVALID_ARGUMENT, "null argument");
  m->model.material.kind = MATERIAL_CALLBACK;
  m->model.material.callback = field;
  m->model.material.user = user;
  return SF_OK;
}

sf_status sf_model_set_shell_core(sf_model* m, sf_material shell, sf_material core, const double lo[3],
                                  const double hi[3], double depth) {
  if (!m || !lo || !hi) return fail(SF_INVALID_ARGUMENT, "null argument");
  MaterialSpec& s = m->model.material;
  s.kind = MATERIAL_SHELL_CORE;
  s.shell = shell;
  s.core = core;
  for (int a = 0; a < 3; ++a) {
    s.lo[a] = lo[a];
    s.hi[a] = hi[a];
  }
  s.depth = depth;
  return SF_OK;
}

sf_status sf_model_set_quadrature(sf_model* m, int32_t rule) {
  if (!m || (rule != SF_QUADRATURE_FOUR_POINT && rule != SF_QUADRATURE_FOURTEEN_POINT))
    return fail(SF_INVALID_ARGUMENT, "unknown quadrature rule");
  m->model.quadrature = rule;
  return SF_OK;
}

sf_status sf_model_fix_node(sf_model* m, uint32_t node) {
  if (!m) return fail(SF_INVALID_ARGUMENT, "null argument");
  m->model.fixed.push_back(node);
  return SF_OK;
}

sf_status sf_model_fix_nodes(sf_model* m, const uint32_t* nodes, uint64_t count) {
  if (!m || (!nodes && count)) return fail(SF_INVALID_ARGUMENT, "null argument");
  m->model.fixed.insert(m->model.fixed.end(), nodes, nodes + count);
  return SF_OK;
}

sf_status sf_model_add_nodal_force(sf_model* m, uint32_t node, const double force[3]) {
  if (!m || !force) return fail(SF_INVALID_ARGUMENT, "null argument");
  m->model.forces.push_back({node, {force[0], force[1], force[2]}});
  return SF_OK;
}

sf_status sf_model_add_traction(sf_model* m, const sf_boundary_face* face, const double traction[3]) {
  if (!m || !face || !traction) return fail(SF_INVALID_ARGUMENT, "null argument");
  m->model.tractions.push_back({*face, {traction[0], traction[1], traction[2]}});
  return SF_OK;
}

sf_status sf_model_add_tractions(sf_model* m, const sf_boundary_face* faces, const double* tractions, uint64_t count) {
  if (!m || ((!faces || !tractions) && count)) return fail(SF_INVALID_ARGUMENT, "null argument");
  for (uint64_t i = 0; i < count; ++i)
    m->model.tractions.push_back({faces[i], {tractions[3 * i], tractions[3 * i + 1], tractions[3 * i + 2]}});
  return SF_OK;
}

sf_status sf_model_prescribe_displacement(sf_model* m, uint32_t node, uint32_t axis, double value) {
  if (!m) return fail(SF_INVALID_ARGUMENT, "null argument");
  for (auto& p : m->model.prescribed)
    if (p.first.first == node && p.first.second == axis) {
      p.second = value;  // the last call for a node and axis wins (study.rs:90-98)
      return SF_OK;
    }
  m->model.prescribed.push_back({{node, axis}, value});
  return SF_OK;
}

void sf_study_options_default(sf_study_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->tolerance = 1e-9;
  o->max_iterations = 0;
  o->preconditioner = SF_PRECONDITIONER_JACOBI;
  o->neighbour_reach = 3.0;
  o->coarse_dofs = 1500;
  o->max_levels = 12;
  o->smoother_degree = 3;
  o->smoother_range = 30.0;
  o->precision = SF_PRECISION_SINGLE_STORAGE;
  o->threads = 0;
  o->device = 0;
  o->use_graphs = 1;
  o->device_memory_budget = 0;
  o->sell_min_rows = 0;
  o->batchable = 0;
  o->coarse_tail = 0;
}

// ------------------------------------------------------------------------------ builder
sf_status sf_builder_create(sf_model* model, const sf_study_options* options, sf_builder** out) {
  std::unique_ptr<sf_model> owned(model);
  if (!model || !options || !out) return fail(SF_INVALID_ARGUMENT, "null argument");
  std::unique_ptr<sf_builder> b(new sf_builder);
  b->model = std::move(model->model);
  b->options = *options;
  b->threads = options->threads ? (int)std::min<uint64_t>(options->threads, 64) : default_threads();
  Model& md = b->model;
  const Mesh& mesh = md.mesh;
  size_t nn = mesh.nodes.size();
  vector<char> is_fixed(nn, 0);
  for (uint32_t n : md.fixed) {
    if (n >= nn) {
      error_slot().node = n;
      return fail(SF_NODE_OUT_OF_RANGE, "a fixed node does not exist");
    }
    is_fixed[n] = 1;
  }
  std::sort(md.prescribed.begin(), md.prescribed.end());
  // The constraint check and the load (StudyBuilder::new's refusals, study.rs:419-474) feed
  // neither the free numbering, the pattern nor the device set-up, so they run on a helper thread
  // while this one builds those; a refusal is returned once both are done, with the helper's
  // error payload, and in the reference's order (constraints, loads, prescribed values).
  vector<double> load(3 * nn, 0.0);
  sf_error helper_error{};
  std::future<sf_status> checks = std::async(std::launch::async, [&]() -> sf_status {
    sf_status st = md.prescribed.empty() ? check_constraints(mesh, is_fixed)
                                         : check_held_dofs(mesh, is_fixed, md.prescribed);
    if (!st) st = build_load(mesh, md, load);
    if (st) helper_error = error_slot();
    return st;
  });
  struct Join {  // the helper reads this frame's vectors: it ends before any return
    std::future<sf_status>& f;
    ~Join() {
      if (f.valid()) f.wait();
    }
  } join{checks};
  b->free.assign(nn, FIXED);
  for (size_t n = 0; n < nn; ++n)
    if (!is_fixed[n]) b->free[n] = (uint32_t)b->free_count++;
  double t0 = now_seconds();
  // A mesh generated on the study's device: the incidence and the pattern are built there too (the
  // same arrays); the host build otherwise, or when a row is too wide for the device build.
  DevicePattern dp;
  bool host_pattern = true;
  if (mesh.dev && mesh.dev->device == b->options.device) {
    if (sf_status e = device_pattern(mesh, b->free, b->free_count, dp, b->pattern.starts, &host_pattern)) return e;
    if (!host_pattern) {
      b->pattern.cols.resize(dp.blocks);
      if (dp.blocks &&
          cudaMemcpy(b->pattern.cols.data(), dp.cols, dp.blocks * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
        release_pattern(mesh.dev->device, dp);
        return cuda_check(cudaGetLastError(), "pattern copy");
      }
    }
  }
  struct DropPattern {  // device pattern arrays not yet handed to the solver are released on a refusal
    DevicePattern& dp;
    int device;
    bool armed = true;
    ~DropPattern() {
      if (armed) release_pattern(device, dp);
    }
  } drop{dp, b->options.device};
  if (host_pattern) build_pattern(mesh, b->free, b->free_count, b->threads, b->pattern);
  if (sf_status st = checks.get()) {
    error_slot() = helper_error;
    return st;
  }
  b->rhs.reserve(3 * b->free_count);
  for (size_t n = 0; n < nn; ++n)
    if (b->free[n] != FIXED)
      for (int a = 0; a < 3; ++a) b->rhs.push_back(load[3 * n + a]);
  for (auto& p : md.prescribed) {
    uint32_t node = p.first.first, axis = p.first.second;
    if (axis > 2) {
      error_slot().axis = axis;
      return fail(SF_AXIS_OUT_OF_RANGE, "an axis other than 0, 1 or 2");
    }
    if (!std::isfinite(p.second)) return fail(SF_NON_FINITE_LOAD, "a prescribed value is not finite");
    if (node >= nn) {
      error_slot().node = node;
      return fail(SF_NODE_OUT_OF_RANGE, "a prescribed node does not exist");
    }
    if (b->free[node] == FIXED) {
      error_slot().node = node;
      return fail(SF_PRESCRIBED_ON_FIXED_NODE, "a prescribed component is on a fixed node");
    }
    b->prescribed.push_back({3 * (size_t)b->free[node] + axis, p.second});
  }
  std::sort(b->prescribed.begin(), b->prescribed.end());
  bool all_zero = true;
  for (double v : b->rhs) all_zero = all_zero && v == 0.0;
  for (auto& p : b->prescribed) all_zero = all_zero && p.second == 0.0;
  if (all_zero) return fail(SF_NO_EFFECTIVE_LOAD, "the model has no effective load");
  // Device set-up: mesh, element stiffness buffer, pattern and assembly map, system matrix.
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(SF_NO_DEVICE, "no CUDA device is visible");
  if (b->options.device < 0 || b->options.device >= ndev) return fail(SF_INVALID_ARGUMENT, "no such CUDA device");
  cudaSetDevice(b->options.device);
  DeviceSolver& s = b->solver;
  s.device = b->options.device;
  s.sell_min_rows = b->options.sell_min_rows ? b->options.sell_min_rows : 32768;
  s.uniform_lanes = b->options.batchable != 0;
  if (s.uniform_lanes) s.sell_min_rows = UINT64_MAX;
  s.coarse_tail = b->options.coarse_tail != 0;
  if (sf_status e = cuda_check(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking), "stream")) return e;
  AssemblyDevice& a = b->asmdev;
  a.tet_count = (uint32_t)mesh.tets.size();
  a.quadrature = md.quadrature;
  a.points = md.quadrature == SF_QUADRATURE_FOURTEEN_POINT ? 14 : 4;
  size_t blocks = b->pattern.cols.size();
  size_t budget = b->options.device_memory_budget;
  const HostPattern& hp = b->pattern;
  const size_t incidence = host_pattern ? hp.inc_start.size() + hp.inc.size() + 2 * hp.row_node.size()
                                        : (nn + 1) + 10 * mesh.tets.size() + 2 * b->free_count;
  size_t need = nn * 24 + mesh.tets.size() * 40 + mesh.tets.size() * 495 * 8 + blocks * (4 + 72) + incidence * 4;
  if (budget && need > budget) return fail(SF_DEVICE_MEMORY_BUDGET, "the assembly does not fit the device memory budget");
  sf_status e = SF_OK;
  if (!e) e = dev_alloc(s, (void**)&a.nodes, nn * 24);
  if (!e) e = dev_alloc(s, (void**)&a.tets, mesh.tets.size() * 40);
  if (!e) e = dev_alloc(s, (void**)&a.ke, mesh.tets.size() * 495 * 8);
  s.system.rows = (uint32_t)b->free_count;
  s.system.rb = s.system.cb = 3;
  s.system.blocks = blocks;
  if (host_pattern) {
    if (!e) e = dev_alloc(s, (void**)&a.inc_start, hp.inc_start.size() * 4);
    if (!e) e = dev_alloc(s, (void**)&a.inc, std::max<size_t>(1, hp.inc.size()) * 4);
    if (!e) e = dev_alloc(s, (void**)&a.row_node, std::max<size_t>(1, hp.row_node.size()) * 4);
    if (!e) e = dev_alloc(s, (void**)&a.cursor, std::max<size_t>(1, hp.row_node.size()) * 4);
    if (!e) e = dev_alloc(s, (void**)&s.system.starts, (b->free_count + 1) * 4);
    if (!e) e = dev_alloc(s, (void**)&s.system.cols, std::max<size_t>(1, blocks) * 4);
  } else {
    // the device-built arrays become the solver's own
    a.inc_start = dp.inc_start;
    a.inc = dp.inc;
    a.row_node = dp.row_node;
    a.cursor = dp.cursor;
    s.system.starts = dp.starts;
    s.system.cols = dp.cols;
    for (auto& al : dp.allocations) {
      s.owned.push_back(al);
      s.bytes += al.second;
    }
    drop.armed = false;
  }
  if (!e) e = dev_alloc(s, (void**)&a.error, 8);
  if (!e) e = dev_alloc(s, &s.system.vals, std::max<size_t>(1, blocks) * 72);
  if (e) {
    release_builder_device(b.get());
    return e;
  }
  if (mesh.dev && mesh.dev->device == s.device) {
    // a mesh generated on this device: its arrays are already here (the solver holds them until
    // it is released, so the copies finish before they can be freed)
    cudaMemcpyAsync(a.nodes, mesh.dev->nodes, nn * 24, cudaMemcpyDeviceToDevice, s.stream);
    cudaMemcpyAsync(a.tets, mesh.dev->tets, mesh.tets.size() * 40, cudaMemcpyDeviceToDevice, s.stream);
    s.mesh_keep = mesh.dev;
  } else {
    copy_h2d(s, a.nodes, mesh.nodes.data(), nn * 24);
    copy_h2d(s, a.tets, mesh.tets.data(), mesh.tets.size() * 40);
  }
  if (host_pattern) {
    // each row's cursor starts at its node's first element
    vector<uint32_t> cursor(hp.row_node.size());
    for (size_t r = 0; r < cursor.size(); ++r) cursor[r] = hp.inc_start[hp.row_node[r]];
    copy_h2d(s, a.inc_start, hp.inc_start.data(), hp.inc_start.size() * 4);
    if (!hp.inc.empty()) copy_h2d(s, a.inc, hp.inc.data(), hp.inc.size() * 4);
    if (!cursor.empty()) {
      copy_h2d(s, a.row_node, hp.row_node.data(), cursor.size() * 4);
      copy_h2d(s, a.cursor, cursor.data(), cursor.size() * 4);
    }
    copy_h2d(s, s.system.starts, b->pattern.starts.data(), (b->free_count + 1) * 4);
    copy_h2d(s, s.system.cols, b->pattern.cols.data(), blocks * 4);
  } else {
    s.d2h_bytes += (b->free_count + 1) * 4 + blocks * 4;  // the pattern's host copy
  }
  unsigned long long none = ~0ull;
  copy_h2d(s, a.error, &none, 8);
  if ((e = make_row_groups(s, s.system, b->pattern.starts.data(), 72))) {
    release_builder_device(b.get());
    return e;
  }
  // A host material callback: integration point positions from the device, the field on the
  // host, (E, nu) per point back to the device.
  if (md.material.kind == MATERIAL_CALLBACK) {
    size_t pts = mesh.tets.size() * a.points;
    e = dev_alloc(s, (void**)&a.positions, pts * 24);
    if (!e) e = dev_alloc(s, (void**)&a.point_material, pts * 16);
    if (!e) e = launch_point_positions(a, s.stream);
    if (e) {
      release_builder_device(b.get());
      return e;
    }
    vector<double> pos(pts * 3);
    copy_d2h(s, pos.data(), a.positions, pts * 24);
    cudaStreamSynchronize(s.stream);
    vector<sf_material> mats(pts);
    md.material.callback(md.material.user, pos.data(), pts, mats.data());
    vector<double> em(pts * 2);
    for (size_t i = 0; i < pts; ++i) {
      em[2 * i] = mats[i].youngs_modulus;
      em[2 * i + 1] = mats[i].poisson_ratio;
    }
    copy_h2d(s, a.point_material, em.data(), pts * 16);
  }
  e = cuda_check(cudaStreamSynchronize(s.stream), "assembly set-up");
  if (e) {
    release_builder_device(b.get());
    return e;
  }
  // The incidence is on the device now.
  vector<uint32_t>().swap(b->pattern.inc_start);
  vector<uint32_t>().swap(b->pattern.inc);
  vector<uint32_t>().swap(b->pattern.row_node);
  b->assembly_seconds = now_seconds() - t0;
  *out = b.release();
  return SF_OK;
}

void sf_builder_destroy(sf_builder* b) {
  if (!b) return;
  // The setup first: it waits for any device work of its own still in flight.
  if (b->setup) setup_destroy(b->setup);
  b->setup = nullptr;
  release_builder_device(b);
  delete b;
}

// StudyBuilder::apply_prescribed (study.rs:564-593) on the device-assembled matrix. Only the
// prescribed block rows and their mirror blocks change, so those blocks are gathered to the host,
// eliminated there in the reference's order, and written back: each prescribed component, by
// ascending DOF, takes its row's off-diagonal entries by ascending column, moves entry x value off
// every unconstrained right-hand side, and zeroes the entry and its transpose; then its own
// right-hand side becomes diagonal x value.
static sf_status apply_prescribed(sf_builder* b) {
  if (b->prescribed.empty() || b->prescribed_applied) return SF_OK;
  b->prescribed_applied = true;
  DeviceSolver& s = b->solver;
  const HostPattern& hp = b->pattern;
  auto find = [&](uint32_t row, uint32_t col) -> uint32_t {
    const uint32_t* lo = hp.cols.data() + hp.starts[row];
    const uint32_t* hi = hp.cols.data() + hp.starts[row + 1];
    return (uint32_t)(std::lower_bound(lo, hi, col) - hp.cols.data());
  };
  std::map<uint32_t, size_t> slot;
  vector<uint32_t> list;
  auto need = [&](uint32_t k) {
    if (slot.emplace(k, list.size()).second) list.push_back(k);
  };
  for (auto& p : b->prescribed) {
    uint32_t r = (uint32_t)(p.first / 3);
    for (uint32_t k = hp.starts[r]; k < hp.starts[r + 1]; ++k) {
      need(k);
      need(find(hp.cols[k], r));
    }
  }
  uint32_t* d_idx = nullptr;
  double* d_vals = nullptr;
  sf_status e = dev_alloc(s, (void**)&d_idx, list.size() * 4);
  if (!e) e = dev_alloc(s, (void**)&d_vals, list.size() * 72);
  vector<double> vals(list.size() * 9);
  if (!e) {
    copy_h2d(s, d_idx, list.data(), list.size() * 4);
    e = setup_gather_blocks(s.stream, list.size(), 9, d_idx, (const double*)s.system.vals, d_vals);
  }
  if (!e) {
    copy_d2h(s, vals.data(), d_vals, vals.size() * 8);
    e = cuda_check(cudaStreamSynchronize(s.stream), "prescribed blocks");
  }
  if (e) return e;
  auto at = [&](size_t i, size_t j) -> double& {
    uint32_t k = find((uint32_t)(i / 3), (uint32_t)(j / 3));
    return vals[slot[k] * 9 + (i % 3) * 3 + j % 3];
  };
  vector<char> constrained(b->rhs.size(), 0);
  for (auto& p : b->prescribed) constrained[p.first] = 1;
  for (auto& p : b->prescribed) {
    const size_t dof = p.first, r = dof / 3, pr = dof % 3;
    const double value = p.second;
    for (uint32_t k = hp.starts[r]; k < hp.starts[r + 1]; ++k)
      for (size_t q = 0; q < 3; ++q) {
        size_t c = 3 * (size_t)hp.cols[k] + q;
        if (c == dof) continue;
        double& entry_ref = vals[slot[k] * 9 + pr * 3 + q];
        double entry = entry_ref;
        if (!constrained[c]) b->rhs[c] -= entry * value;
        at(c, dof) += -entry;
        entry_ref += -entry;
      }
  }
  for (auto& p : b->prescribed) b->rhs[p.first] = at(p.first, p.first) * p.second;
  copy_h2d(s, d_vals, vals.data(), vals.size() * 8);
  e = setup_scatter_blocks(s.stream, list.size(), 9, d_idx, d_vals, (double*)s.system.vals);
  if (!e) e = cuda_check(cudaStreamSynchronize(s.stream), "prescribed blocks");
  dev_free(s, d_idx);
  dev_free(s, d_vals);
  return e;
}

static sf_status builder_assemble(sf_builder* b, uint64_t max_elements, sf_cancel_fn cancel, void* user) {
  size_t total = b->model.mesh.tets.size();
  if (b->next >= total) return SF_OK;
  if (cancel && cancel(user)) {
    b->failure = SF_CANCELLED;
    return fail(SF_CANCELLED, "assembly was cancelled");
  }
  size_t end = (size_t)std::min<uint64_t>(total, b->next + std::max<uint64_t>(max_elements, 1));
  DeviceSolver& s = b->solver;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, s.stream);
  sf_status st = launch_element_stiffness(b->asmdev, b->model.material, (uint32_t)b->next, (uint32_t)end, s.stream);
  if (!st) st = launch_gather(b->asmdev, s.system, (uint32_t)end, s.stream);
  s.launches += 2;
  cudaEventRecord(e1, s.stream);
  if (!st) st = cuda_check(cudaStreamSynchronize(s.stream), "assembly");
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  b->assembly_ms += ms;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st) return st;
  unsigned long long err = 0;
  cudaMemcpy(&err, b->asmdev.error, 8, cudaMemcpyDeviceToHost);
  if (err != ~0ull) {
    error_slot().tet = (uint32_t)(err >> 32);
    error_slot().point = (uint32_t)((err >> 8) & 0xff);
    b->failure = (err & 0xff) == FAULT_INVERTED ? SF_ELEMENT_INVERTED_JACOBIAN : SF_ELEMENT_INVALID_MATERIAL;
    return fail(b->failure, (err & 0xff) == FAULT_INVERTED ? "an element's Jacobian is inverted at an integration point"
                                                           : "the material at an integration point is not a stable solid");
  }
  b->next = end;
  if (end == total) {
    if (sf_status pe = apply_prescribed(b)) {
      b->failure = pe;
      return pe;
    }
    AssemblyDevice& a = b->asmdev;
    if (b->options.preconditioner == SF_PRECONDITIONER_MULTIGRID) {
      // The near-null modes, from the free rows' nodes while the row map is still on the device,
      // zero at prescribed DOFs (the setup reads them at the tentative prolongator).
      double center[3], scale = 1.0;
      rigid_frame(b->model.mesh.nodes, b->free, b->free_count, center, &scale);
      sf_status me = dev_alloc(s, (void**)&b->modes, std::max<size_t>(1, b->free_count) * 18 * 8);
      if (!me) me = setup_rigid_modes(s.stream, (uint32_t)b->free_count, a.row_node, a.nodes, center, scale, b->modes);
      if (!me && !b->prescribed.empty()) {
        vector<uint32_t> idx;
        for (auto& p : b->prescribed)
          for (uint32_t k = 0; k < 6; ++k) idx.push_back((uint32_t)(p.first * 6 + k));
        vector<double> zeros(idx.size(), 0.0);
        uint32_t* d_idx = nullptr;
        double* d_zero = nullptr;
        me = dev_alloc(s, (void**)&d_idx, idx.size() * 4);
        if (!me) me = dev_alloc(s, (void**)&d_zero, zeros.size() * 8);
        if (!me) {
          copy_h2d(s, d_idx, idx.data(), idx.size() * 4);
          copy_h2d(s, d_zero, zeros.data(), zeros.size() * 8);
          me = setup_set_values(s.stream, idx.size(), d_idx, d_zero, b->modes);
        }
        if (!me) me = cuda_check(cudaStreamSynchronize(s.stream), "near-null modes");
        dev_free(s, d_idx);
        dev_free(s, d_zero);
      }
      if (me) {
        b->failure = me;
        return me;
      }
    }
    // The element stiffness buffer and the assembly map have served; free them for the solve.
    for (void* p : {(void*)a.ke, (void*)a.inc_start, (void*)a.inc, (void*)a.row_node, (void*)a.cursor})
      dev_free(s, p);
    a.ke = nullptr;
    a.inc_start = a.inc = a.row_node = a.cursor = nullptr;
  }
  return SF_OK;
}

static sf_status builder_setup(sf_builder* b, uint64_t budget, sf_cancel_fn cancel, void* user) {
  if (b->setup_finished) return SF_OK;
  double t0 = now_seconds();
  if (!b->setup) {
    // The fine level as setup reads it: the device-assembled f64 blocks.
    DeviceSolver& s = b->solver;
    Bsr fine;
    fine.rows = b->free_count;
    fine.rb = fine.cb = 3;
    fine.starts = b->pattern.starts;
    fine.cols.assign(b->pattern.cols.begin(), b->pattern.cols.end());
    fine.dev = (double*)s.system.vals;
    fine.dev_starts = s.system.starts;
    fine.dev_cols = s.system.cols;
    vector<P3> positions;
    positions.reserve(b->free_count);
    for (size_t n = 0; n < b->free.size(); ++n)
      if (b->free[n] != FIXED) positions.push_back(b->model.mesh.nodes[n]);
    SetupOptions so;
    so.reach = b->options.neighbour_reach;
    so.coarse_dofs = b->options.coarse_dofs;
    so.max_levels = b->options.max_levels;
    so.range = b->options.smoother_range;
    so.threads = b->threads;
    b->setup = setup_create(s, std::move(fine), vector<double>(), std::move(positions), so, b->modes);
    b->modes = nullptr;  // the setup frees it
  }
  bool finished = false;
  sf_status st = setup_step(b->setup, budget, cancel, user, &finished);
  b->preconditioner_seconds += now_seconds() - t0;
  if (st) {
    b->failure = st;
    return st;
  }
  b->setup_finished = finished;
  return SF_OK;
}

sf_status sf_builder_step(sf_builder* b, uint64_t max_elements, sf_cancel_fn cancel, void* user, sf_build_progress* p) {
  if (!b) return fail(SF_INVALID_ARGUMENT, "null argument");
  if (b->failure) return fail(b->failure, "the build failed earlier");
  cudaSetDevice(b->solver.device);
  double t0 = now_seconds();
  sf_status st = builder_assemble(b, max_elements, cancel, user);
  b->assembly_seconds += now_seconds() - t0;
  if (st) return st;
  size_t total = b->model.mesh.tets.size();
  if (b->next == total && b->options.preconditioner == SF_PRECONDITIONER_MULTIGRID) {
    st = builder_setup(b, max_elements, cancel, user);
    if (st) return st;
  }
  if (p) {
    p->elements_done = b->next;
    p->elements_total = total;
    p->setup_finished = b->next == total && (b->options.preconditioner != SF_PRECONDITIONER_MULTIGRID || b->setup_finished);
  }
  return SF_OK;
}

static void fill_stats(sf_study* s) {
  if (s->levels.empty()) return;
  bool single = s->solver.storage_single;
  size_t sb = single ? 4 : 8;
  auto values = [](const Bsr& m) { return m.cols.size() * m.rb * m.cb; };
  double finest = (double)values(s->levels[0].a);
  size_t stored = 0, memory = 0;
  for (auto& lv : s->levels) {
    stored += values(lv.a);
    memory += (lv.a.starts.size()) * 8 + lv.a.cols.size() * 4 + values(lv.a) * sb;
    memory += lv.a.rows * lv.a.rb * lv.a.rb * sb;
    if (lv.has_p) memory += lv.p.starts.size() * 8 + lv.p.cols.size() * 4 + values(lv.p) * sb;
    if (lv.has_factor) memory += lv.factor_n * lv.factor_n * 8;
  }
  s->report.has_multigrid = 1;
  s->report.mg_levels = s->levels.size();
  s->report.mg_coarse_dofs = s->levels.back().a.rows * s->levels.back().a.rb;
  s->report.mg_operator_complexity = (double)stored / finest;
  s->report.mg_memory_bytes = memory;
}

sf_status sf_builder_finish(sf_builder* b, sf_study** out) {
  if (!b || !out) return fail(SF_INVALID_ARGUMENT, "null argument");
  if (b->failure) return fail(b->failure, "the build failed earlier");
  bool mg = b->options.preconditioner == SF_PRECONDITIONER_MULTIGRID;
  if (b->next != b->model.mesh.tets.size() || (mg && !b->setup_finished))
    return fail(SF_NOT_FINISHED, "elements or setup remain");
  cudaSetDevice(b->solver.device);
  double t0 = now_seconds();
  std::unique_ptr<sf_study> s(new sf_study);
  s->model = std::move(b->model);
  s->options = b->options;
  s->free = std::move(b->free);
  s->free_count = b->free_count;
  s->rhs = std::move(b->rhs);
  s->prescribed = std::move(b->prescribed);
  s->pattern = std::move(b->pattern);
  s->asmdev = b->asmdev;
  s->solver = b->solver;
  b->solver = DeviceSolver();
  DeviceSolver& d = s->solver;
  d.n = (uint32_t)(3 * s->free_count);
  d.multigrid = mg;
  int prec = s->options.precision;
  d.precision = prec;
  d.storage_single = prec != SF_PRECISION_DOUBLE;
  d.vector_single = prec == SF_PRECISION_SINGLE || prec == SF_PRECISION_MIXED;
  d.flexible = prec == SF_PRECISION_MIXED;
  sf_status e = SF_OK;
  double** vecs[] = {&d.rhs, &d.x, &d.r, &d.z, &d.p, &d.ap};
  for (double** v : vecs)
    if (!e) e = dev_alloc(d, (void**)v, (size_t)d.n * 8);
  if (!e) e = dev_alloc(d, (void**)&d.partials, kReduceBlocks * 4 * 8);
  if (!e) e = dev_alloc(d, (void**)&d.state, sizeof(PcgState));
  if (!e) e = dev_alloc(d, (void**)&d.always_active, sizeof(int));
  if (e) return e;
  copy_h2d(d, d.rhs, s->rhs.data(), (size_t)d.n * 8);
  // The conjugate gradient's f64 product runs on a SELL copy when the system has many rows.
  if (wants_sell(d.system, d.sell_min_rows))
    if ((e = make_sell_from_device(d, d.system, s->pattern.starts.data(), s->pattern.cols.data()))) return e;
  if (mg) {
    s->levels = setup_take_levels(b->setup);
    e = solver_upload_hierarchy(d, s->levels, s->options.smoother_degree);
    if (e) return e;
    fill_stats(s.get());
  } else {
    // Jacobi (preconditioner.rs:221-234): the inverse of the positive diagonal.
    vector<double> diag(d.n);
    vector<double> vals(s->pattern.cols.size() * 9);
    copy_d2h(d, vals.data(), d.system.vals, vals.size() * 8);
    cudaStreamSynchronize(d.stream);
    for (size_t r = 0; r < s->free_count; ++r) {
      const uint32_t* cb = s->pattern.cols.data() + s->pattern.starts[r];
      const uint32_t* ce = s->pattern.cols.data() + s->pattern.starts[r + 1];
      size_t at = std::lower_bound(cb, ce, (uint32_t)r) - s->pattern.cols.data();
      for (int i = 0; i < 3; ++i) {
        double v = vals[at * 9 + i * 3 + i];
        if (std::isnan(v) || v <= 0.0 || !std::isfinite(v)) {
          error_slot().row = 3 * r + i;
          error_slot().value = v;
          return fail(SF_JACOBI_DIAGONAL, "a diagonal entry is not positive");
        }
        diag[3 * r + i] = 1.0 / v;
      }
    }
    if ((e = dev_alloc(d, (void**)&d.jacobi, (size_t)d.n * 8))) return e;
    copy_h2d(d, d.jacobi, diag.data(), (size_t)d.n * 8);
    cudaStreamSynchronize(d.stream);
  }
  if (s->options.device_memory_budget && d.bytes > s->options.device_memory_budget)
    return fail(SF_DEVICE_MEMORY_BUDGET, "the study does not fit the device memory budget");
  e = solver_init_pcg(d, s->options.tolerance, s->options.max_iterations);
  if (!e) e = cuda_check(cudaStreamSynchronize(d.stream), "solver init");
  if (e) return e;
  if (s->options.use_graphs) {
    if ((e = solver_capture_graph(d))) return e;
  }
  s->pinned = (PcgState*)pinned_slot();
  if (!s->pinned) return fail(SF_CUDA_ERROR, "cudaMallocHost failed");
  cudaEventCreate(&s->ev0);
  cudaEventCreate(&s->ev1);
  std::memset(&s->report, 0, sizeof(s->report));
  fill_stats(s.get());
  s->report.total_dofs = 3 * s->model.mesh.nodes.size();
  s->report.free_dofs = 3 * s->free_count;
  s->report.nonzeros = s->pattern.cols.size() * 9;
  s->report.relative_residual = 1.0;
  s->report.assembly_seconds = b->assembly_seconds + (now_seconds() - t0);
  s->report.preconditioner_seconds = b->preconditioner_seconds;
  s->assembly_ms = b->assembly_ms;
  solver_read_state(d, &s->last);
  s->status = s->last.status;
  *out = s.release();
  delete b;
  return SF_OK;
}

sf_status sf_study_create(sf_model* model, const sf_study_options* options, sf_cancel_fn cancel, void* user,
                          sf_study** out) {
  sf_builder* b = nullptr;
  if (sf_status e = sf_builder_create(model, options, &b)) return e;
  sf_build_progress p;
  sf_status e = sf_builder_step(b, UINT64_MAX, cancel, user, &p);
  if (!e) e = sf_builder_finish(b, out);
  if (e) {
    sf_builder_destroy(b);
    return e;
  }
  return SF_OK;
}

// ------------------------------------------------------------------------------ solve
static void fill_progress(const PcgState& st, sf_progress* p) {
  p->iteration = st.iterations;
  p->relative_residual = st.rel;
  p->at_rounding_floor = st.at_floor;
}

}  // extern "C"

namespace sf {

// Pcg::step (pcg.rs:167-190) on the device: up to max_iterations iterations, enqueued in chunks;
// every kernel of an iteration after the solve ends returns at once, so the state is read back
// once per chunk, with one chunk in flight ahead. `cancel` is read before every iteration.
sf_status run_iterations(DeviceSolver& d, bool use_graphs, uint64_t max_iterations, sf_cancel_fn cancel, void* user,
                         PcgState* pinned, PcgState& last, int& status, bool& cancelled) {
  uint64_t done = 0;
  const uint64_t chunk_max = 16;
  uint64_t chunk = 4;
  bool stop = false;
  while (!stop && done < max_iterations) {
    uint64_t k = std::min<uint64_t>(chunk, max_iterations - done);
    uint64_t launched = 0;
    for (; launched < k; ++launched) {
      if (cancel && cancel(user)) {
        cancelled = true;
        stop = true;
        break;
      }
      sf_status e = SF_OK;
      if (use_graphs) {
        e = cuda_check(cudaGraphLaunch(d.graph_exec, d.stream), "graph launch");
        d.launches += d.graph_kernels;
      } else {
        e = solver_enqueue_iteration(d);
        d.launches += d.launches_per_iteration;
      }
      if (e) return e;
    }
    done += launched;
    copy_d2h(d, pinned, d.state, sizeof(PcgState));
    if (sf_status e = cuda_check(cudaStreamSynchronize(d.stream), "solver step")) return e;
    last = *pinned;
    status = last.status;
    if (status != ST_ACTIVE) stop = true;
    chunk = std::min(chunk_max, chunk * 2);
  }
  return SF_OK;
}

// The StepOutcome of a step that ended with `status` (pcg.rs:47-57, 216-275): the kind and the
// progress, and for a failed solve its PcgError as the returned status with its payload.
sf_status step_result(int status, bool cancelled, const PcgState& last, sf_step_outcome* out) {
  if (out) {
    out->kind = cancelled ? SF_OUTCOME_CANCELLED : status == ST_CONVERGED ? SF_OUTCOME_CONVERGED : SF_OUTCOME_RUNNING;
    fill_progress(last, &out->progress);
  }
  if (cancelled) return SF_OK;
  if (status == ST_FAILED_NOT_PD) {
    error_slot().iteration = last.fail_iteration;
    error_slot().curvature = last.curvature;
    return fail(SF_PCG_NOT_POSITIVE_DEFINITE, "the system is not positive definite along the search direction");
  }
  if (status == ST_FAILED_NOT_CONVERGED) {
    error_slot().iteration = last.iterations;
    error_slot().relative_residual = last.rel;
    return fail(SF_PCG_NOT_CONVERGED, "the iteration cap ran out before the tolerance");
  }
  return SF_OK;
}

}  // namespace sf

extern "C" {

sf_status sf_study_step(sf_study* s, uint64_t max_iterations, sf_cancel_fn cancel, void* user, sf_step_outcome* out) {
  if (!s) return fail(SF_INVALID_ARGUMENT, "null argument");
  DeviceSolver& d = s->solver;
  cudaSetDevice(d.device);
  auto finish = [&]() -> sf_status {
    s->report.iterations = s->last.iterations;
    s->report.relative_residual = s->last.rel;
    s->report.at_rounding_floor = s->last.at_floor;
    return step_result(s->status, s->cancelled, s->last, out);
  };
  if (s->cancelled || s->status != ST_ACTIVE) return finish();
  double t0 = now_seconds();
  cudaEventRecord(s->ev0, d.stream);
  if (sf_status e = run_iterations(d, s->options.use_graphs != 0, max_iterations, cancel, user, s->pinned, s->last,
                                   s->status, s->cancelled))
    return e;
  cudaEventRecord(s->ev1, d.stream);
  cudaEventSynchronize(s->ev1);
  float ms = 0;
  cudaEventElapsedTime(&ms, s->ev0, s->ev1);
  s->step_ms = ms;
  s->report.solve_seconds += now_seconds() - t0;
  return finish();
}

/* Pcg::progress (pcg.rs:200-207) of a study's solve. */
sf_status sf_study_progress(const sf_study* s, sf_progress* out) {
  if (!s || !out) return fail(SF_INVALID_ARGUMENT, "null argument");
  fill_progress(s->last, out);
  return SF_OK;
}

}  // extern "C"

namespace sf {

BatchRunner::~BatchRunner() {
  batch_destroy(it);
  for (void* p : slots) pinned_release(p);
  if (stream) cudaStreamDestroy(stream);
}

sf_status BatchRunner::init(int dev) {
  device = dev;
  cudaSetDevice(dev);
  return cuda_check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "batch stream");
}

sf_status BatchRunner::rebuild() {
  batch_destroy(it);
  dirty = false;
  if (members.empty()) return SF_OK;
  std::vector<DeviceSolver*> inst;
  for (sf_study* m : members) inst.push_back(&m->solver);
  while (slots.size() < members.size()) {
    void* p = pinned_slot();
    if (!p) return fail(SF_CUDA_ERROR, "cudaMallocHost failed");
    slots.push_back(p);
  }
  return batch_build(inst, stream, it);
}

sf_status BatchRunner::run_chunk(uint64_t iterations, std::vector<sf_study*>& finished) {
  cudaSetDevice(device);
  if (dirty)
    if (sf_status e = rebuild()) return e;
  if (members.empty()) return SF_OK;
  double t0 = now_seconds();
  if (sf_status e = batch_replay(it, iterations)) return e;
  for (size_t i = 0; i < members.size(); ++i) {
    cudaMemcpyAsync(slots[i], members[i]->solver.state, sizeof(PcgState), cudaMemcpyDeviceToHost, stream);
    members[i]->solver.d2h_bytes += sizeof(PcgState);
    members[i]->solver.launches += it.sites * iterations;
  }
  if (sf_status e = cuda_check(cudaStreamSynchronize(stream), "batch chunk")) return e;
  double dt = now_seconds() - t0;
  std::vector<sf_study*> keep;
  for (size_t i = 0; i < members.size(); ++i) {
    sf_study* m = members[i];
    m->last = *(const PcgState*)slots[i];
    m->status = m->last.status;
    m->report.solve_seconds += dt;
    m->report.iterations = m->last.iterations;
    m->report.relative_residual = m->last.rel;
    m->report.at_rounding_floor = m->last.at_floor;
    if (m->status == ST_ACTIVE)
      keep.push_back(m);
    else
      finished.push_back(m);
  }
  if (keep.size() != members.size()) {
    members.swap(keep);
    dirty = true;
  }
  return SF_OK;
}

uint64_t study_signature(sf_study* s) {
  std::vector<LaunchRecord> rec;
  g_recorder = &rec;
  sf_status e = solver_enqueue_iteration(s->solver);
  g_recorder = nullptr;
  if (e) return 0;
  uint64_t h = 1469598103934665603ull;
  auto mix = [&](uint64_t v) {
    for (int i = 0; i < 8; ++i) {
      h ^= (v >> (8 * i)) & 0xff;
      h *= 1099511628211ull;
    }
  };
  for (auto& r : rec) {
    mix((uint64_t)(uintptr_t)r.batched);
    mix(r.pack.size());
  }
  mix(s->solver.device);
  return h;
}

uint64_t study_device_bytes(const sf_study* s) { return s->solver.bytes; }

uint64_t model_free_dofs(const sf_model* m) {
  std::vector<uint32_t> fixed = m->model.fixed;
  std::sort(fixed.begin(), fixed.end());
  fixed.erase(std::unique(fixed.begin(), fixed.end()), fixed.end());
  size_t nodes = m->model.mesh.nodes.size();
  size_t held = 0;
  for (uint32_t n : fixed) held += n < nodes ? 1 : 0;
  return 3 * (nodes - held);
}

uint64_t model_node_count(const sf_model* m) { return m->model.mesh.nodes.size(); }

// The outcome and status of a study that left a batch.
static sf_status batch_outcome(sf_study* m, sf_step_outcome* out) {
  if (out) {
    out->kind = m->status == ST_CONVERGED ? SF_OUTCOME_CONVERGED : SF_OUTCOME_RUNNING;
    fill_progress(m->last, &out->progress);
  }
  if (m->status == ST_FAILED_NOT_PD) return SF_PCG_NOT_POSITIVE_DEFINITE;
  if (m->status == ST_FAILED_NOT_CONVERGED) return SF_PCG_NOT_CONVERGED;
  return SF_OK;
}

}  // namespace sf

extern "C" {

sf_status sf_study_solve_batch(sf_study** studies, uint64_t count, sf_step_outcome* outcomes, sf_status* statuses) {
  if (!studies || count == 0) return fail(SF_INVALID_ARGUMENT, "an empty batch");
  for (uint64_t i = 0; i < count; ++i) {
    if (!studies[i]) return fail(SF_INVALID_ARGUMENT, "null study");
    if (studies[i]->solver.device != studies[0]->solver.device)
      return fail(SF_INVALID_ARGUMENT, "the studies of a batch must share their device");
    for (uint64_t j = 0; j < i; ++j)
      if (studies[j] == studies[i]) return fail(SF_INVALID_ARGUMENT, "a study appears twice in a batch");
  }
  BatchRunner run;
  if (sf_status e = run.init(studies[0]->solver.device)) return e;
  for (uint64_t i = 0; i < count; ++i) {
    if (sf_status e = sf_study_resolve(studies[i], nullptr)) return e;
    if (sf_status e = cuda_check(cudaStreamSynchronize(studies[i]->solver.stream), "batch start")) return e;
    run.members.push_back(studies[i]);
  }
  std::vector<sf_study*> finished;
  uint64_t chunk = 4;
  while (!run.members.empty()) {
    if (sf_status e = run.run_chunk(chunk, finished)) return e;
    chunk = std::min<uint64_t>(16, chunk * 2);
  }
  for (uint64_t i = 0; i < count; ++i) {
    sf_status st = batch_outcome(studies[i], outcomes ? outcomes + i : nullptr);
    if (statuses) statuses[i] = st;
  }
  return SF_OK;
}

sf_status sf_study_displacements(const sf_study* s, double* out) {
  if (!s || !out) return fail(SF_INVALID_ARGUMENT, "null argument");
  const DeviceSolver& d = s->solver;
  vector<double> x(d.n);
  cudaSetDevice(d.device);
  copy_d2h(d, x.data(), d.x, (size_t)d.n * 8);
  if (sf_status e = cuda_check(cudaStreamSynchronize(d.stream), "read displacements")) return e;
  for (size_t n = 0; n < s->free.size(); ++n)
    for (int a = 0; a < 3; ++a) out[3 * n + a] = s->free[n] == FIXED ? 0.0 : x[3 * (size_t)s->free[n] + a];
  // A prescribed component is exact, not the solver's estimate of it (study.rs:233-236).
  for (auto& p : s->model.prescribed) out[3 * (size_t)p.first.first + p.first.second] = p.second;
  return SF_OK;
}

sf_status sf_study_report(const sf_study* s, sf_report* out) {
  if (!s || !out) return fail(SF_INVALID_ARGUMENT, "null argument");
  *out = s->report;
  return SF_OK;
}

// Device stress recovery (Recovery, results.rs:97-124, 376-539). The incidence lists every
// recovery of a study reads are built once on the host; a recovery snapshots the displacements on
// the device and advances in the reference's units of work (each element, then each vertex's
// patch fit); the nodal field is made when both are done.
static sf_status recovery_tables(sf_study* s) {
  RecoveryDevice& r = s->rec;
  if (r.ready) return SF_OK;
  DeviceSolver& d = s->solver;
  const Mesh& m = s->model.mesh;
  const size_t nn = m.nodes.size(), ne = m.tets.size(), nv = m.vertex_count;
  // Elements touching each vertex through a corner, and (element, local node) per node, both in
  // element order (results.rs:414-435); the first element reaching each midside node.
  vector<uint32_t> voff(nv + 1, 0), noff(nn + 1, 0);
  for (auto& t : m.tets) {
    for (int c = 0; c < 4; ++c) voff[t[c] + 1] += 1;
    for (int a = 0; a < 10; ++a) noff[t[a] + 1] += 1;
  }
  for (size_t i = 0; i < nv; ++i) voff[i + 1] += voff[i];
  for (size_t i = 0; i < nn; ++i) noff[i + 1] += noff[i];
  vector<uint32_t> vinc(voff[nv]), ninc(noff[nn]);
  vector<uint32_t> vf(voff.begin(), voff.end() - 1), nf(noff.begin(), noff.end() - 1);
  vector<uint32_t> mid(nn - nv, 0xffffffffu);
  for (size_t e = 0; e < ne; ++e) {
    const auto& t = m.tets[e];
    for (int c = 0; c < 4; ++c) vinc[vf[t[c]]++] = (uint32_t)e;
    for (int a = 0; a < 10; ++a) ninc[nf[t[a]]++] = ((uint32_t)e << 4) | (uint32_t)a;
    for (int k = 0; k < 6; ++k)
      if (mid[t[4 + k] - nv] == 0xffffffffu) mid[t[4 + k] - nv] = ((uint32_t)e << 3) | (uint32_t)k;
  }
  sf_status e = SF_OK;
  if (!e) e = dev_alloc(d, (void**)&r.free, nn * 4);
  if (!e) e = dev_alloc(d, (void**)&r.vertex_offsets, (nv + 1) * 4);
  if (!e) e = dev_alloc(d, (void**)&r.vertex_incident, std::max<size_t>(1, vinc.size()) * 4);
  if (!e) e = dev_alloc(d, (void**)&r.node_offsets, (nn + 1) * 4);
  if (!e) e = dev_alloc(d, (void**)&r.node_incident, std::max<size_t>(1, ninc.size()) * 4);
  if (!e) e = dev_alloc(d, (void**)&r.midside_first, std::max<size_t>(1, mid.size()) * 4);
  if (e) return e;
  copy_h2d(d, r.free, s->free.data(), nn * 4);
  copy_h2d(d, r.vertex_offsets, voff.data(), voff.size() * 4);
  if (!vinc.empty()) copy_h2d(d, r.vertex_incident, vinc.data(), vinc.size() * 4);
  copy_h2d(d, r.node_offsets, noff.data(), noff.size() * 4);
  if (!ninc.empty()) copy_h2d(d, r.node_incident, ninc.data(), ninc.size() * 4);
  if (!mid.empty()) copy_h2d(d, r.midside_first, mid.data(), mid.size() * 4);
  if ((e = cuda_check(cudaStreamSynchronize(d.stream), "recovery set-up"))) return e;
  r.ready = true;
  return SF_OK;
}

static void recovery_free(sf_recovery* r) {
  if (!r) return;
  if (sf_study* s = r->study) {
    DeviceSolver& d = s->solver;
    cudaSetDevice(d.device);
    cudaStreamSynchronize(d.stream);
    for (void* p : r->owned) dev_free(d, p);
    s->recoveries.erase(std::remove(s->recoveries.begin(), s->recoveries.end(), r), s->recoveries.end());
  }
  delete r;
}

// Recovery::new (results.rs:103-124) on the device: a snapshot of the current displacements
// (prescribed components exact, fixed nodes zero) and the buffers of the work to come.
static sf_status recovery_begin(sf_study* s, sf_recovery** out) {
  if (sf_status e = recovery_tables(s)) return e;
  DeviceSolver& d = s->solver;
  const Mesh& m = s->model.mesh;
  const size_t nn = m.nodes.size(), ne = m.tets.size(), nv = m.vertex_count;
  const size_t pts = (size_t)s->asmdev.points * ne;
  std::unique_ptr<sf_recovery> rec(new sf_recovery);
  rec->study = s;
  rec->converged = s->status == ST_CONVERGED;
  RecoveryDevice& r = rec->dev;
  r = s->rec;  // the shared tables
  auto alloc = [&](void** p, size_t bytes) -> sf_status {
    if (sf_status e = dev_alloc(d, p, std::max<size_t>(bytes, 8))) return e;
    rec->owned.push_back(*p);
    return SF_OK;
  };
  sf_status e = SF_OK;
  if (!e) e = alloc((void**)&r.disp, nn * 24);
  if (!e) e = alloc((void**)&r.point_stress, pts * 48);
  if (!e) e = alloc((void**)&r.point_vm, pts * 8);
  if (!e) e = alloc((void**)&r.point_pos, pts * 24);
  if (!e) e = alloc((void**)&r.point_mat, pts * 16);
  if (!e) e = alloc((void**)&r.node_candidate, ne * 10 * 56);
  if (!e) e = alloc((void**)&r.fits, nv * 28 * 8);
  if (!e) e = alloc((void**)&r.has_fit, nv * 4);
  if (!e) e = alloc((void**)&r.nodal_stress, nn * 48);
  if (!e) e = alloc((void**)&r.nodal_vm, nn * 8);
  if (!e) e = launch_scatter_displacements(d.x, r, (uint32_t)nn, d.stream);
  if (!e && !s->model.prescribed.empty()) {
    // the prescribed components, exact
    vector<uint32_t> idx;
    vector<double> val;
    for (auto& p : s->model.prescribed) {
      idx.push_back(3 * p.first.first + p.first.second);
      val.push_back(p.second);
    }
    uint32_t* d_idx = nullptr;
    double* d_val = nullptr;
    e = dev_alloc(d, (void**)&d_idx, idx.size() * 4);
    if (!e) e = dev_alloc(d, (void**)&d_val, val.size() * 8);
    if (!e) {
      copy_h2d(d, d_idx, idx.data(), idx.size() * 4);
      copy_h2d(d, d_val, val.data(), val.size() * 8);
      e = setup_set_values(d.stream, idx.size(), d_idx, d_val, r.disp);
    }
    if (!e) e = cuda_check(cudaStreamSynchronize(d.stream), "recovery snapshot");
    dev_free(d, d_idx);
    dev_free(d, d_val);
  }
  d.launches += 1;
  s->recoveries.push_back(rec.get());
  if (e) {
    recovery_free(rec.release());
    return e;
  }
  *out = rec.release();
  return SF_OK;
}

// Recovery::advance (results.rs:470-539): up to `budget` more units, elements first, then patch
// fits; `cancel` is read before each launch. Returns the element fault the reference would name.
static sf_status recovery_advance(sf_study* s, sf_recovery* rec, uint64_t budget, sf_cancel_fn cancel, void* user) {
  DeviceSolver& d = s->solver;
  const uint64_t ne = s->model.mesh.tets.size(), nv = s->model.mesh.vertex_count;
  double t0 = now_seconds();
  sf_status e = SF_OK;
  if (rec->next_element < ne && budget > 0) {
    if (cancel && cancel(user)) return fail(SF_CANCELLED, "the recovery was cancelled");
    const uint64_t end = std::min<uint64_t>(ne, rec->next_element + budget);
    unsigned long long none = ~0ull, err = 0;
    copy_h2d(d, s->asmdev.error, &none, 8);
    e = launch_recovery_elements(s->asmdev, s->model.material, rec->dev, (uint32_t)rec->next_element, (uint32_t)end,
                                 d.stream);
    d.launches += 1;
    if (!e) copy_d2h(d, &err, s->asmdev.error, 8);
    if (!e) e = cuda_check(cudaStreamSynchronize(d.stream), "recovery");
    if (e) return e;
    if (err != ~0ull) {
      error_slot().tet = (uint32_t)(err >> 32);
      error_slot().point = (uint32_t)((err >> 8) & 0xff);
      return fail((err & 0xff) == FAULT_INVERTED ? SF_ELEMENT_INVERTED_JACOBIAN : SF_ELEMENT_INVALID_MATERIAL,
                  "recovery met an inverted element or an invalid material");
    }
    budget -= end - rec->next_element;
    rec->next_element = end;
  }
  if (rec->next_element == ne && rec->next_vertex < nv && budget > 0) {
    if (cancel && cancel(user)) return fail(SF_CANCELLED, "the recovery was cancelled");
    const uint64_t end = std::min<uint64_t>(nv, rec->next_vertex + budget);
    e = launch_recovery_fits(s->asmdev, rec->dev, (uint32_t)rec->next_vertex, (uint32_t)end, d.stream);
    d.launches += 1;
    if (!e) e = cuda_check(cudaStreamSynchronize(d.stream), "recovery");
    if (e) return e;
    rec->next_vertex = end;
  }
  s->report.recovery_seconds += now_seconds() - t0;
  return SF_OK;
}

static bool recovery_finished(const sf_study* s, const sf_recovery* r) {
  return r->next_element == s->model.mesh.tets.size() && r->next_vertex == s->model.mesh.vertex_count;
}

// Recovery::into_field (results.rs:376-410) and the copies out: any output may be null.
static sf_status recovery_outputs(sf_study* s, sf_recovery* rec, double* displacements, double* nodal_stress,
                                  double* nodal_von_mises, sf_point_stress* points) {
  DeviceSolver& d = s->solver;
  const Mesh& m = s->model.mesh;
  const size_t nn = m.nodes.size(), ne = m.tets.size();
  const size_t q = (size_t)s->asmdev.points, pts = q * ne;
  sf_status e = launch_recovery_field(s->asmdev, rec->dev, (uint32_t)nn, (uint32_t)m.vertex_count, d.stream);
  d.launches += 1;
  if (e) return e;
  if (displacements) copy_d2h(d, displacements, rec->dev.disp, nn * 24);
  if (nodal_stress) copy_d2h(d, nodal_stress, rec->dev.nodal_stress, nn * 48);
  if (nodal_von_mises) copy_d2h(d, nodal_von_mises, rec->dev.nodal_vm, nn * 8);
  vector<double> ps, pv, pp;
  if (points) {
    ps.resize(pts * 6);
    pv.resize(pts);
    pp.resize(pts * 3);
    copy_d2h(d, ps.data(), rec->dev.point_stress, pts * 48);
    copy_d2h(d, pv.data(), rec->dev.point_vm, pts * 8);
    copy_d2h(d, pp.data(), rec->dev.point_pos, pts * 24);
  }
  if ((e = cuda_check(cudaStreamSynchronize(d.stream), "read recovery"))) return e;
  if (points)
    for (size_t i = 0; i < pts; ++i) {
      points[i].tet = (uint32_t)(i / q);
      points[i].point = (uint32_t)(i % q);
      for (int k = 0; k < 3; ++k) points[i].position[k] = pp[i * 3 + k];
      for (int k = 0; k < 6; ++k) points[i].stress[k] = ps[i * 6 + k];
      points[i].von_mises = pv[i];
    }
  return SF_OK;
}

// Units of recovery work per launch when the caller gives no budget (sf_study_solution): the
// cancel callback is read between such slices.
static const uint64_t kRecoverySlice = 1u << 16;

sf_status sf_study_solution(sf_study* s, sf_cancel_fn cancel, void* user, double* displacements,
                            double* nodal_stress, double* nodal_von_mises, sf_point_stress* points) {
  if (!s) return fail(SF_INVALID_ARGUMENT, "null argument");
  if (s->status != ST_CONVERGED) return fail(SF_NOT_FINISHED, "the solve has not converged");
  DeviceSolver& d = s->solver;
  cudaSetDevice(d.device);
  if (!nodal_stress && !nodal_von_mises && !points) return sf_study_displacements(s, displacements);
  if (!s->answer) {
    sf_recovery* rec = nullptr;
    if (sf_status e = recovery_begin(s, &rec)) return e;
    while (!recovery_finished(s, rec)) {
      if (sf_status e = recovery_advance(s, rec, kRecoverySlice, cancel, user)) {
        recovery_free(rec);
        return e;
      }
    }
    s->answer = rec;
  }
  return recovery_outputs(s, s->answer, displacements, nodal_stress, nodal_von_mises, points);
}

sf_status sf_study_begin_recovery(sf_study* s, sf_recovery** out) {
  if (!s || !out) return fail(SF_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  cudaSetDevice(s->solver.device);
  return recovery_begin(s, out);
}

sf_status sf_study_continue_recovery(sf_study* s, sf_recovery* r, uint64_t max_units, sf_cancel_fn cancel, void* user,
                                     int32_t* finished) {
  if (!s || !r || r->study != s) return fail(SF_INVALID_ARGUMENT, "a recovery of another study");
  cudaSetDevice(s->solver.device);
  sf_status e = recovery_advance(s, r, max_units, cancel, user);
  if (finished) *finished = recovery_finished(s, r) ? 1 : 0;
  return e;
}

sf_status sf_study_finish_recovery(sf_study* s, sf_recovery* r, double* displacements, double* nodal_stress,
                                   double* nodal_von_mises, sf_point_stress* points) {
  if (!s || !r || r->study != s) return fail(SF_INVALID_ARGUMENT, "a recovery of another study");
  if (!recovery_finished(s, r)) return fail(SF_NOT_FINISHED, "elements or patch fits remain");
  cudaSetDevice(s->solver.device);
  return recovery_outputs(s, r, displacements, nodal_stress, nodal_von_mises, points);
}

void sf_recovery_destroy(sf_recovery* r) { recovery_free(r); }

void sf_study_destroy(sf_study* s) { delete s; }

// ------------------------------------------------------------------------------ inspection
sf_status sf_study_matrix(const sf_study* s, uint64_t* row_starts, uint32_t* columns, double* values) {
  if (!s || !row_starts || !columns || !values) return fail(SF_INVALID_ARGUMENT, "null argument");
  const DeviceSolver& d = s->solver;
  size_t blocks = s->pattern.cols.size();
  vector<double> vals(blocks * 9);
  cudaSetDevice(d.device);
  copy_d2h(d, vals.data(), d.system.vals, blocks * 72);
  if (sf_status e = cuda_check(cudaStreamSynchronize(d.stream), "read matrix")) return e;
  // Scalar CSR rows from 3x3 blocks: row 3R + i holds block columns in order, three each.
  uint64_t at = 0;
  row_starts[0] = 0;
  for (size_t r = 0; r < s->free_count; ++r)
    for (int i = 0; i < 3; ++i) {
      for (uint32_t b = s->pattern.starts[r]; b < s->pattern.starts[r + 1]; ++b)
        for (int k = 0; k < 3; ++k) {
          columns[at] = 3 * s->pattern.cols[b] + k;
          values[at] = vals[(size_t)b * 9 + i * 3 + k];
          ++at;
        }
      row_starts[3 * r + i + 1] = at;
    }
  return SF_OK;
}

sf_status sf_study_rhs(const sf_study* s, double* out) {
  if (!s || !out) return fail(SF_INVALID_ARGUMENT, "null argument");
  std::memcpy(out, s->rhs.data(), s->rhs.size() * 8);
  return SF_OK;
}

uint64_t sf_study_level_count(const sf_study* s) { return s ? s->levels.size() : 0; }

sf_status sf_study_level_info(const sf_study* s, uint64_t level, sf_level_info* out) {
  if (!s || !out || level >= s->levels.size()) return fail(SF_INVALID_ARGUMENT, "no such level");
  const HostLevel& lv = s->levels[level];
  out->rows = lv.a.rows;
  out->row_block = lv.a.rb;
  out->blocks = lv.a.cols.size();
  out->lambda_min = lv.lambda_min;
  out->lambda_max = lv.lambda_max;
  out->has_prolongator = lv.has_p;
  out->prolongator_blocks = lv.has_p ? lv.p.cols.size() : 0;
  out->has_factor = lv.has_factor;
  return SF_OK;
}

sf_status sf_study_level_matrix(const sf_study* s, uint64_t level, int32_t prolongator, uint64_t* starts,
                                uint32_t* columns, double* values) {
  if (!s || level >= s->levels.size() || !starts || !columns || !values) return fail(SF_INVALID_ARGUMENT, "no such level");
  const HostLevel& lv = s->levels[level];
  if (prolongator && !lv.has_p) return fail(SF_INVALID_ARGUMENT, "the coarsest level has no prolongator");
  const Bsr& m = prolongator ? lv.p : lv.a;
  for (size_t i = 0; i <= m.rows; ++i) starts[i] = m.starts[i];
  std::memcpy(columns, m.cols.data(), m.cols.size() * 4);
  size_t n = m.cols.size() * m.rb * m.cb;
  if (n == 0) return SF_OK;
  cudaSetDevice(s->solver.device);
  copy_d2h(s->solver, values, m.dev, n * 8);
  return cuda_check(cudaStreamSynchronize(s->solver.stream), "level values");
}

sf_status sf_study_aggregates(const sf_study* s, uint64_t level, uint32_t* out) {
  if (!s || level >= s->levels.size() || !out) return fail(SF_INVALID_ARGUMENT, "no such level");
  const HostLevel& lv = s->levels[level];
  std::memcpy(out, lv.aggregates.data(), lv.aggregates.size() * 4);
  return SF_OK;
}

sf_status sf_study_precondition(sf_study* s, const double* residual, double* output) {
  if (!s || !residual || !output) return fail(SF_INVALID_ARGUMENT, "null argument");
  DeviceSolver& d = s->solver;
  cudaSetDevice(d.device);
  double *din = nullptr, *dout = nullptr;
  if (sf_status e = cuda_check(cudaMalloc((void**)&din, (size_t)d.n * 8 + 64), "cudaMalloc")) return e;
  if (sf_status e = cuda_check(cudaMalloc((void**)&dout, (size_t)d.n * 8 + 64), "cudaMalloc")) {
    cudaFree(din);
    return e;
  }
  copy_h2d(d, din, residual, (size_t)d.n * 8);
  sf_status e = solver_precondition(d, din, dout);
  if (!e) {
    copy_d2h(d, output, dout, (size_t)d.n * 8);
    e = cuda_check(cudaStreamSynchronize(d.stream), "precondition");
  }
  cudaFree(din);
  cudaFree(dout);
  return e;
}

sf_status sf_study_level_stage(sf_study* s, uint64_t level, int32_t stage, const double* in0, const double* in1,
                               double* out0, double* out1) {
  if (!s || !in0 || !out0) return fail(SF_INVALID_ARGUMENT, "null argument");
  DeviceSolver& d = s->solver;
  if (!d.multigrid || level >= d.levels.size()) return fail(SF_INVALID_ARGUMENT, "no such multigrid level");
  const bool two_in = stage == SF_STAGE_SMOOTH_ADD || stage == SF_STAGE_RESIDUAL || stage == SF_STAGE_PROLONG ||
                      stage == SF_STAGE_RESIDUAL_START;
  const bool two_out = stage == SF_STAGE_RESTRICT_START || stage == SF_STAGE_RESIDUAL_START;
  if ((two_in && !in1) || (two_out && !out1)) return fail(SF_INVALID_ARGUMENT, "null argument");
  const bool has_coarse = level + 1 < d.levels.size();
  const size_t n = d.levels[level].n, cn = has_coarse ? d.levels[level + 1].n : 0;
  // lengths: the coarse level's for the prolongation's e and the restrictions' outputs
  const size_t n_in0 = stage == SF_STAGE_PROLONG ? cn : n;
  const size_t n_out = stage == SF_STAGE_RESTRICT || stage == SF_STAGE_RESTRICT_START ? cn : n;
  if ((n_in0 == 0 || n_out == 0)) return fail(SF_INVALID_ARGUMENT, "the level has no coarser level");
  cudaSetDevice(d.device);
  double *di0 = nullptr, *di1 = nullptr, *do0 = nullptr, *do1 = nullptr;
  sf_status e = dev_alloc(d, (void**)&di0, n_in0 * 8);
  if (!e) e = dev_alloc(d, (void**)&di1, n * 8);
  if (!e) e = dev_alloc(d, (void**)&do0, n_out * 8);
  if (!e) e = dev_alloc(d, (void**)&do1, n_out * 8);
  if (!e) {
    copy_h2d(d, di0, in0, n_in0 * 8);
    if (two_in) copy_h2d(d, di1, in1, n * 8);
    e = solver_level_stage(d, level, stage, di0, di1, do0, do1);
  }
  if (!e) {
    copy_d2h(d, out0, do0, n_out * 8);
    if (two_out) copy_d2h(d, out1, do1, n_out * 8);
    e = cuda_check(cudaStreamSynchronize(d.stream), "level stage");
  }
  for (double* p : {di0, di1, do0, do1}) dev_free(d, p);
  return e;
}

sf_status sf_study_system_multiply(sf_study* s, const double* x, double* y) {
  if (!s || !x || !y) return fail(SF_INVALID_ARGUMENT, "null argument");
  DeviceSolver& d = s->solver;
  cudaSetDevice(d.device);
  double *din = nullptr, *dout = nullptr;
  if (sf_status e = cuda_check(cudaMalloc((void**)&din, (size_t)d.n * 8 + 64), "cudaMalloc")) return e;
  if (sf_status e = cuda_check(cudaMalloc((void**)&dout, (size_t)d.n * 8 + 64), "cudaMalloc")) {
    cudaFree(din);
    return e;
  }
  copy_h2d(d, din, x, (size_t)d.n * 8);
  sf_status e = solver_system_multiply(d, din, dout);
  if (!e) {
    copy_d2h(d, y, dout, (size_t)d.n * 8);
    e = cuda_check(cudaStreamSynchronize(d.stream), "system multiply");
  }
  cudaFree(din);
  cudaFree(dout);
  return e;
}

namespace {
typedef CUresult (*AddressRangeFn)(CUdeviceptr*, size_t*, CUdeviceptr);

// The driver's cuMemGetAddressRange, looked up through the runtime (the library does not link the
// driver library itself); null where the driver does not offer it.
AddressRangeFn address_range_fn() {
  static AddressRangeFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuMemGetAddressRange", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return (AddressRangeFn) nullptr;
    }
    return (AddressRangeFn)f;
  }();
  return fn;
}

// `bytes` of device (or managed) memory of the study's device from p, aligned for doubles and
// inside one allocation, so a kernel given the range stays in bounds.
bool on_study_device(const void* p, size_t bytes, int device) {
  if ((uintptr_t)p % alignof(double) != 0) return false;
  cudaPointerAttributes attr{};
  if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (attr.type != cudaMemoryTypeManaged && !(attr.type == cudaMemoryTypeDevice && attr.device == device))
    return false;
  AddressRangeFn range = address_range_fn();
  if (!range) return false;
  CUdeviceptr base = 0;
  size_t size = 0;
  if (range(&base, &size, (CUdeviceptr)(uintptr_t)p) != CUDA_SUCCESS) return false;
  return (uintptr_t)p + bytes <= (uintptr_t)base + size;
}
bool overlaps(const void* a, size_t abytes, const void* b, size_t bbytes) {
  uintptr_t a0 = (uintptr_t)a, b0 = (uintptr_t)b;
  return a0 < b0 + bbytes && b0 < a0 + abytes;
}
}  // namespace

sf_status sf_study_energy_products(sf_study* s, const double* x, double* y, double* energy, uint64_t count) {
  if (!s) return fail(SF_INVALID_ARGUMENT, "null study");
  DeviceSolver& d = s->solver;
  if (count > solver_energy_max_vectors()) return solver_energy_products(d, x, y, energy, count);
  if (count == 0) return SF_OK;
  if (!x || !y || !energy) return fail(SF_INVALID_ARGUMENT, "null argument");
  // The caller's current device is put back on every return.
  int caller_device = 0;
  if (sf_status e = cuda_check(cudaGetDevice(&caller_device), "cudaGetDevice")) return e;
  struct Restore {
    int device;
    ~Restore() { cudaSetDevice(device); }
  } restore{caller_device};
  if (sf_status e = cuda_check(cudaSetDevice(d.device), "cudaSetDevice")) return e;
  const size_t vbytes = (size_t)count * d.n * sizeof(double), ebytes = (size_t)count * sizeof(double);
  if (!on_study_device(x, vbytes, d.device) || !on_study_device(y, vbytes, d.device) ||
      !on_study_device(energy, ebytes, d.device))
    return fail(SF_INVALID_ARGUMENT, "x, y and energy must be 8-byte aligned device memory of the study's device, "
                                     "each range inside one allocation");
  if (overlaps(x, vbytes, y, vbytes) || overlaps(x, vbytes, energy, ebytes) || overlaps(y, vbytes, energy, ebytes))
    return fail(SF_INVALID_ARGUMENT, "x, y and energy must not overlap");
  return solver_energy_products(d, x, y, energy, count);
}

sf_status sf_study_device_timing(const sf_study* s, sf_device_timing* out) {
  if (!s || !out) return fail(SF_INVALID_ARGUMENT, "null argument");
  out->step_ms = s->step_ms;
  out->assembly_ms = s->assembly_ms;
  out->setup_ms = 0;
  out->kernel_launches = s->solver.launches;
  out->h2d_bytes = s->solver.h2d_bytes;
  out->d2h_bytes = s->solver.d2h_bytes;
  out->launches_per_iteration = s->solver.launches_per_iteration;
  out->coarse_tail_level = s->solver.tail_level;
  out->coarse_tail_cluster = s->solver.tail_cluster;
  return SF_OK;
}

sf_status sf_study_resolve(sf_study* s, const double* rhs) {
  if (!s) return fail(SF_INVALID_ARGUMENT, "null argument");
  DeviceSolver& d = s->solver;
  cudaSetDevice(d.device);
  if (rhs) {
    std::memcpy(s->rhs.data(), rhs, (size_t)d.n * 8);
    copy_h2d(d, d.rhs, rhs, (size_t)d.n * 8);
  }
  if (sf_status e = solver_restart(d, s->options.tolerance, s->options.max_iterations)) return e;
  s->release_answer();
  s->cancelled = false;
  std::memset(&s->last, 0, sizeof(s->last));
  s->status = ST_ACTIVE;
  s->report.iterations = 0;
  s->report.relative_residual = 1.0;
  s->report.at_rounding_floor = 0;
  return SF_OK;
}

uint64_t sf_study_stream(const sf_study* s) { return s ? (uint64_t)(uintptr_t)s->solver.stream : 0; }

sf_status sf_study_time_kernel(sf_study* s, int32_t kernel, uint64_t repeats, sf_kernel_timing* out) {
  if (!s || !out) return fail(SF_INVALID_ARGUMENT, "null argument");
  cudaSetDevice(s->solver.device);
  double ms = 0, bytes = 0;
  if (sf_status e = solver_time_kernel(s->solver, kernel, repeats, &ms, &bytes)) return e;
  out->ms_per_launch = ms;
  out->bytes_per_launch = bytes;
  out->launches = repeats;
  return SF_OK;
}

}  // extern "C"
