// Internal host-side types of solidfem_b200: the mesh, the model, the multigrid setup's block
// matrices and the study state. Device buffers and kernels are declared in device.h.
#pragma once

#include <array>
#include <cstdint>
#include <cstring>
#include <functional>
#include <string>
#include <memory>
#include <utility>
#include <vector>

#include "../../include/solidfem_b200.h"

namespace sf {

using std::array;
using std::size_t;
using std::vector;
typedef array<double, 3> P3;

static const uint32_t FIXED = 0xffffffffu;
static const uint32_t NO_AGGREGATE = 0xffffffffu;

// Local node indices of each face (crates/solidfem-mesh/src/boundary.rs:8-13) and the corner pair
// of each edge midpoint (crates/solidfem-mesh/src/quadratic.rs:10).
extern const int kFaceNodes[4][6];
extern const int kEdgeCorners[6][2];

// ----------------------------------------------------------------------------- errors
// Records a failure for sf_last_error and returns its status.
sf_status fail(sf_status status, const char* message);
sf_error& error_slot();

// ----------------------------------------------------------------------------- mesh
// The ten-node arrays of a mesh built on a device, kept there for the studies made from it (a
// study on the same device copies them device to device instead of uploading the host arrays).
struct DeviceMesh {
  int device = 0;
  double* nodes = nullptr;   // node_count x 3
  uint32_t* tets = nullptr;  // tet_count x 10
  virtual ~DeviceMesh() {}
};

struct Mesh {
  vector<P3> nodes;
  vector<array<uint32_t, 10>> tets;
  vector<array<uint32_t, 4>> corners;
  size_t vertex_count = 0;
  vector<sf_boundary_face> faces;  // sorted by their sorted corners
  std::shared_ptr<DeviceMesh> dev;  // set when the mesh was built on a device
};

sf_status build_box_mesh(const double origin[3], const double size[3], const uint64_t div[3],
                         Mesh& out);
sf_status build_linear_mesh(const double* positions, uint64_t n, const uint32_t* tets,
                            uint64_t ntets, Mesh& out);
vector<vector<uint32_t>> face_connected_bodies(const Mesh& mesh);
// The same meshes built on a CUDA device (mesh_device.cu), bit-identical to the host builders;
// `out.dev` keeps the ten-node arrays on the device.
sf_status build_box_mesh_device(const double origin[3], const double size[3], const uint64_t div[3], int device,
                                Mesh& out);
sf_status build_linear_mesh_device(const double* positions, uint64_t n, const uint32_t* tets, uint64_t ntets,
                                   int device, Mesh& out);
// The demo's part grid (demo/wasm/src/part.rs:135-189): grid lines per axis (counts[a] lines),
// the cells of the hollow core dropped when wall_cells > 0.
sf_status build_part_mesh_device(const double* const lines[3], const uint64_t counts[3], uint64_t wall_cells,
                                 int device, Mesh& out);
// build_pattern on the device of a generated mesh: the node-to-element incidence (each node's
// elements ascending), each free row's node and assembly cursor, and the block pattern (starts and
// sorted columns) in device arrays the caller takes over (`allocations`: pointer and bytes of each,
// from the device's stream-ordered pool), the row starts also on the host. *fallback is set, and
// nothing kept, when a row has too many candidate columns for the device build.
struct DevicePattern {
  uint32_t* inc_start = nullptr;  // node_count + 1
  uint32_t* inc = nullptr;        // 10 x tet_count
  uint32_t* row_node = nullptr;   // free rows
  uint32_t* cursor = nullptr;     // free rows
  uint32_t* starts = nullptr;     // free rows + 1
  uint32_t* cols = nullptr;       // blocks
  size_t blocks = 0;
  vector<std::pair<void*, size_t>> allocations;
};
sf_status device_pattern(const Mesh& mesh, const vector<uint32_t>& free, size_t free_count, DevicePattern& out,
                         vector<uint32_t>& host_starts, bool* fallback);
// build_load's consistent traction sums (loads.rs:10-41) on the device of a generated mesh, added
// to the nodal-force sums already in `load`, in the host's order (the same bits).
sf_status device_traction_load(const Mesh& mesh, const vector<std::pair<sf_boundary_face, array<double, 3>>>& tractions,
                               vector<double>& load);

// ----------------------------------------------------------------------------- model
enum MaterialKind { MATERIAL_UNIFORM = 0, MATERIAL_SHELL_CORE = 1, MATERIAL_CALLBACK = 2 };

struct MaterialSpec {
  int kind = MATERIAL_UNIFORM;
  sf_material uniform{0, 0};
  sf_material shell{0, 0}, core{0, 0};
  double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  double depth = 0;
  sf_material_field_fn callback = nullptr;
  void* user = nullptr;
};

struct Model {
  Mesh mesh;
  MaterialSpec material;
  int quadrature = SF_QUADRATURE_FOUR_POINT;
  vector<uint32_t> fixed;  // as given; deduplicated when the builder starts
  vector<std::pair<uint32_t, array<double, 3>>> forces;
  vector<std::pair<sf_boundary_face, array<double, 3>>> tractions;
  vector<std::pair<std::pair<uint32_t, uint32_t>, double>> prescribed;  // (node, axis) -> value
};

// ----------------------------------------------------------------------------- block CSR
// A block sparse matrix of dense rb x cb row-major blocks, f64 (setup works in f64). The pattern
// is on the host; the multigrid levels keep their values on the device (`dev`, with device
// copies of the pattern), and `vals` is filled on the host only where host code reads values.
struct Bsr {
  size_t rows = 0, rb = 0, cb = 0;
  vector<uint32_t> starts;  // rows + 1
  vector<uint32_t> cols;
  vector<double> vals;
  double* dev = nullptr;            // blocks * rb * cb f64 values on the device
  uint32_t* dev_starts = nullptr;   // device copies of starts and cols
  uint32_t* dev_cols = nullptr;
  size_t blocks() const { return cols.size(); }
  size_t block_len() const { return rb * cb; }
  const double* block(size_t at) const { return vals.data() + at * rb * cb; }
  double* block(size_t at) { return vals.data() + at * rb * cb; }
};

// One finished level of the hierarchy: host patterns, f64 values on the device as setup built them.
struct HostLevel {
  Bsr a;
  double* inverse_diagonal = nullptr;  // device, rows * rb * rb f64
  double lambda_min = 0, lambda_max = 0;
  bool has_p = false;
  Bsr p;
  bool has_factor = false;
  size_t factor_n = 0;
  double* dev_coarse_inverse = nullptr;  // the dense inverse of the coarsest level, row-major f64, device
  vector<uint32_t> aggregates;
};

struct SetupOptions {
  double reach = 3.0;
  size_t coarse_dofs = 1500;
  size_t max_levels = 12;
  double range = 30.0;
  int threads = 1;
};

// The multigrid setup (crates/solidfem-solve/src/multigrid/setup.rs) over the device-assembled
// fine level (`fine` carries the host pattern and the device values and pattern). Graph phases
// run on the host, numeric phases on the solver's device and stream; every allocation belongs to
// the solver. Resumable by phase, like the reference's state machine.
struct SetupMachine;
struct DeviceSolver;
// The finest level's near-null modes come either from the host (`near_null`, 6 per scalar row) or,
// when `device_near_null` is set, already on the device (owned by the solver; the setup frees it
// once the tentative prolongator is built).
SetupMachine* setup_create(DeviceSolver& solver, Bsr&& fine, vector<double>&& near_null, vector<P3>&& positions,
                           const SetupOptions& options, double* device_near_null = nullptr);
// Runs up to `budget` rows of work. Returns SF_OK and sets *finished, or a failure.
sf_status setup_step(SetupMachine* machine, size_t budget, sf_cancel_fn cancel, void* user,
                     bool* finished);
vector<HostLevel> setup_take_levels(SetupMachine* machine);
void setup_destroy(SetupMachine* machine);

int default_threads();
double now_seconds();

}  // namespace sf
