// Device-side data of a study and the host launchers of the sm_100a kernels. Kernels live in
// assembly.cu (bit-exact FP64 assembly and recovery, built with -fmad=false) and solve.cu (the
// solve path: block SpMV, Chebyshev smoother, transfers, coarse solve, PCG with fixed-order
// reductions).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "sf_internal.h"

namespace sf {

// A block sparse matrix on the device: rows x (rb x cb) row-major blocks of S values.
struct DevBsr {
  uint32_t rows = 0, rb = 0, cb = 0;
  size_t blocks = 0;
  uint32_t* starts = nullptr;  // rows + 1
  uint32_t* cols = nullptr;    // blocks
  void* vals = nullptr;        // blocks * rb * cb values of the storage type
  // Row groups: runs of consecutive rows whose value slab fits a warp's staging buffer. A warp
  // streams one group into shared memory while it multiplies the previous one.
  uint4* groups = nullptr;     // per group {first row, end row, first block, end block}
  uint32_t ngroups = 0;
  uint32_t group_bytes = 0;    // the largest group's value bytes
  uint32_t group_blocks = 0;   // the largest group's block count
  uint32_t group_rows = 0;     // the largest group's row count
  int lanes_per_row = 32;      // lanes sharing one row: 32, 16, 8 or 4
  // SELL-32 copy for operators with many rows: slices of 32 rows (rows sorted by block count
  // inside windows of kSellWindow rows), one thread per row. Each lane reads its row in chunks of
  // U = sell_chunk_blocks(rb * cb, value bytes) consecutive blocks, 144 bytes of values stored as
  // nine 16-byte vectors: chunk c of slice s starts at block Q0 = slice_start[s] + 32 U c; lane t's
  // columns are cols[Q0 + U t ..], and value i (= u * rb * cb + e of its u-th block) sits at
  // vals[Q0 * rb * cb + (i / VEC) * 32 VEC + t VEC + i % VEC] with VEC values per 16 bytes, so each
  // vector load of a warp is 512 contiguous bytes. Slice widths are padded to whole chunks.
  bool sell = false;
  // Split-row copy (operators of 6-row blocks with many rows): the same slices, but each block
  // row takes six lanes, one per scalar row, and a slice holds kSplitRowsPerSlice block rows
  // (lanes 6 m .. 6 m + 5; lanes 30 and 31 idle). Lane t = 6 m + p reads row p of each block, so
  // its "blocks" are 1 x cb: values as in SELL-32 with block length cb, U = sell_chunk_blocks(cb,
  // value bytes). Columns are stored once per block row: chunk c of slice s keeps them at
  // cols[(slice_start[s] / 32) * 5 + 5 U c + U m ..] for the six lanes of block row m to share.
  bool split = false;
  uint32_t nslices = 0;
  uint32_t* sell_rows = nullptr;   // nslices * 32: the row of each lane (rows when padding)
  uint32_t* sell_len = nullptr;    // nslices * 32: its block count
  uint32_t* sell_start = nullptr;  // nslices + 1, in blocks
  uint32_t* sell_cols = nullptr;
  void* sell_vals = nullptr;
};

static const uint32_t kSellWindow = 2048;    // rows are sorted by length inside windows this long
static const uint32_t kSplitRowsPerSlice = 5;  // block rows of six scalar rows per 32-lane slice
static const uint32_t kSplitMinRows = 4096;    // 6-row block operators with this many rows split

// Blocks per SELL lane chunk: 144 bytes of values, at least one block.
constexpr int sell_chunk_blocks(int len, int value_bytes) {
  return len * value_bytes >= 144 ? 1 : 144 / (len * value_bytes);
}
// Where value e of the block in SELL slot q (a column index position) lives.
__host__ __device__ inline size_t sell_value_offset(size_t q, int len, int chunk, int vec, int e) {
  const size_t r = q % (32u * (size_t)chunk);
  const size_t t = r / (size_t)chunk, u = r % (size_t)chunk;
  const size_t i = u * (size_t)len + (size_t)e;
  return (q - r) * (size_t)len + (i / (size_t)vec) * 32u * (size_t)vec + t * (size_t)vec + i % (size_t)vec;
}

// The SELL copy of a matrix whose values live only on the device (the assembled f64 system):
// the layout from host starts/columns, the values permuted on the device.
sf_status make_sell_from_device(struct DeviceSolver& s, DevBsr& m, const uint32_t* starts, const uint32_t* cols);

// Shared memory one warp of the row-group engine may stage (two groups); the launch opts in to
// 200 KB per block.
static const size_t kMaxStagePerWarp = 192 * 1024;
// True when an operator runs in the SELL-32 layout: many rows, or a row group too long to stage.
bool wants_sell(const DevBsr& m, uint64_t sell_min_rows);
// True when an operator of 6-row blocks runs split, one lane per scalar row: enough block rows
// to fill the device with six lanes each (level 1 of an elasticity hierarchy and the transpose
// restricting onto it), and launches whose kernel may depend on the size (not batchable).
bool wants_split(const DevBsr& m, bool uniform_lanes);

// Splits the rows of a block matrix into groups of at most `target` value bytes (a longer row is
// a group of its own) and chooses the lanes per row from the mean blocks per row.
sf_status make_row_groups(struct DeviceSolver& s, DevBsr& m, const uint32_t* host_starts, size_t value_bytes);

// The solver's scalar state, resident on the device so the iteration loop runs without host
// round trips; kernels read `status` and exit early once the solve has ended.
enum { ST_ACTIVE = 0, ST_CONVERGED = 1, ST_FAILED_NOT_PD = 2, ST_FAILED_NOT_CONVERGED = 3 };
enum { MODE_NORMAL = 0, MODE_CHECK = 1, MODE_RESTART = 2 };

struct PcgState {
  double rz, alpha, beta, curvature, rel, rhs_norm, tolerance, floor;
  double partial_rz, partial_apz;
  unsigned long long iterations, max_iterations, fail_iteration;
  int status, mode, at_floor, flexible;
  unsigned int tickets[8];
};

// Reduction scratch: one partial per block of the fixed reduction grid.
static const int kReduceBlocks = 592;  // 4 x 148 SMs
static const int kReduceThreads = 256;

struct DevLevel {
  DevBsr a;          // the level operator in storage precision
  void* dinv = nullptr;  // rows * rb * rb, storage precision
  DevBsr p;          // prolongator to the next level (rb x 6), storage precision
  DevBsr r;          // its explicit transpose (6 x rb), for gather restriction
  bool has_p = false;
  bool has_factor = false;
  uint32_t n = 0;         // scalar rows
  double* coarse_inverse = nullptr;  // n x n f64, coarsest factored level
  // Chebyshev scalars in f64 (ChebyshevCoefficients, gpu/layout.rs:443-465)
  double theta = 0;
  std::vector<std::pair<double, double>> steps;
  // vectors of the vector precision
  void *b = nullptr, *x = nullptr, *res = nullptr, *z = nullptr, *d0 = nullptr, *d1 = nullptr,
       *post_x = nullptr, *tmp = nullptr;
};

struct DeviceSolver {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::shared_ptr<DeviceMesh> mesh_keep;  // a device-generated mesh whose arrays were copied on `stream`
  int precision = SF_PRECISION_SINGLE_STORAGE;
  bool storage_single = true, vector_single = false, flexible = false;
  bool multigrid = false;
  uint32_t n = 0;  // free dofs
  DevBsr system;   // f64 3x3 system matrix
  double *rhs = nullptr, *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *ap = nullptr;
  float* z32 = nullptr;  // the cycle's f32 output when the cycle runs in f32
  double* jacobi = nullptr;
  double* partials = nullptr;   // kReduceBlocks * 4
  PcgState* state = nullptr;
  int* always_active = nullptr;  // a status word fixed at ST_ACTIVE for standalone cycles
  std::vector<DevLevel> levels;
  std::vector<std::pair<void*, size_t>> owned;  // every cudaMalloc of this solver, with its size
  size_t bytes = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  uint64_t launches_per_iteration = 0;
  uint64_t graph_kernels = 0;     // kernel nodes in the captured iteration graph
  uint64_t launches = 0;          // kernels launched so far (graph replays count their kernels)
  mutable uint64_t h2d_bytes = 0, d2h_bytes = 0;
  uint64_t sell_min_rows = 32768;  // operators with at least this many rows use SELL-32
  bool uniform_lanes = false;      // lanes per row by block shape alone (batchable studies)
  bool coarse_tail = false;        // fuse the last smoothed level and the coarse solve when they fit
  int tail_level = -1;             // the level whose cycle runs as one cluster launch, or -1
  unsigned tail_cluster = 0;       // CTAs of that cluster
  size_t tail_smem = 0;            // shared memory of each of its CTAs
};

// One recorded kernel launch: the batched form of the kernel, its launch shape and the bytes of its
// argument pack. While `g_recorder` is set on a thread, solve launches on that thread are recorded
// instead of executed (batch construction).
struct LaunchRecord {
  const void* batched = nullptr;
  dim3 grid, block;
  size_t smem = 0;
  unsigned cluster = 0;  // CTAs per thread-block cluster (grid.x), 0 for a plain launch
  std::vector<unsigned char> pack;
};
extern thread_local std::vector<LaunchRecord>* g_recorder;

// ------------------------------------------------------------------- memory helpers
// Stream-ordered copies that count the bytes crossing the host-device link.
inline void copy_h2d(const DeviceSolver& s, void* dst, const void* src, size_t bytes) {
  cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s.stream);
  __atomic_fetch_add(&s.h2d_bytes, bytes, __ATOMIC_RELAXED);  // setup's helper thread copies too
}
inline void copy_d2h(const DeviceSolver& s, void* dst, const void* src, size_t bytes) {
  cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s.stream);
  __atomic_fetch_add(&s.d2h_bytes, bytes, __ATOMIC_RELAXED);
}
// Pinned host memory that is never freed (freeing pinned memory synchronizes the device):
// pooled buffers, and 512-byte slots for per-study state.
static const size_t kPinnedSlotBytes = 512;
// A process-wide pool of page-locked host buffers that are never freed (cudaFreeHost would
// synchronize the whole device): pinned_acquire returns the smallest free buffer of at least
// `bytes` (or a new one), pinned_return hands it back. Unlike the per-thread scratch, a buffer
// belongs to its holder until it is returned, so it may live across resumable steps.
void* pinned_acquire(size_t bytes);
void pinned_return(void* buffer);
void* pinned_slot();
void pinned_release(void* slot);
static_assert(2 * sizeof(PcgState) <= kPinnedSlotBytes, "a slot holds two solver states");

sf_status dev_alloc(DeviceSolver& s, void** ptr, size_t bytes);
// Frees one allocation of dev_alloc before the solver ends (setup temporaries).
void dev_free(DeviceSolver& s, void* ptr);
void dev_free_all(DeviceSolver& s);
sf_status cuda_check(cudaError_t e, const char* what);
// Once per device: the stream-ordered pool keeps freed memory and reserves a first slab.
void pool_setup(int device);

// ------------------------------------------------------------------- setup (setup_device.cu)
// FP64 numeric phases of the multigrid setup, bit-identical to the reference's serial loops.
// Patterns (starts, cols) are device copies of the host-built patterns; values are f64.
sf_status setup_inverse_diagonal(cudaStream_t st, uint32_t rows, int rb, const uint32_t* starts, const uint32_t* cols,
                                 const double* vals, double* inv, unsigned long long* bad, double* pivots);
sf_status setup_block_norms(cudaStream_t st, size_t blocks, int len, const double* vals, double* out);
// One power step s2 = D^-1 (A v), and v = src / d.
sf_status setup_power_step(cudaStream_t st, uint32_t rows, int rb, const uint32_t* starts, const uint32_t* cols,
                           const double* vals, const double* inv, const double* v, double* s2);
sf_status setup_scale(cudaStream_t st, size_t n, const double* src, double d, double* v);
sf_status setup_entry_rows(cudaStream_t st, uint32_t rows, const uint32_t* starts, uint32_t* out);
// The geometric strength graph (aggregate.rs:53-69): with out_starts null, each row's strong count
// into out and its closest squared distance into closest; else the strong columns at out_starts.
sf_status setup_strength(cudaStream_t st, uint32_t rows, const uint32_t* starts, const uint32_t* cols, const double* pos,
                         double limit_scale, double* closest, const uint32_t* out_starts, uint32_t* out);
// One pass of a union pattern (symbolic product): out_starts null counts each row's distinct
// columns into out[row]; otherwise writes them, ascending, at out[out_starts[row] ..]. Columns
// are below `width`.
sf_status setup_union_rows(cudaStream_t st, uint32_t rows, uint32_t width, const uint32_t* outer_starts,
                           const uint32_t* outer_idx, bool self, const uint32_t* inner_starts,
                           const uint32_t* inner_cols, const uint32_t* out_starts, uint32_t* out);
// Listed blocks of len values out of / back into a block array; out[idx[i]] = vals[i].
sf_status setup_gather_blocks(cudaStream_t st, size_t count, int len, const uint32_t* idx, const double* in,
                              double* out);
sf_status setup_scatter_blocks(cudaStream_t st, size_t count, int len, const uint32_t* idx, const double* in,
                               double* out);
sf_status setup_set_values(cudaStream_t st, size_t count, const uint32_t* idx, const double* vals, double* out);
// The free nodes' rigid-body modes (rows x 3 x 6) about `center`, scaled (rigid_modes.rs:36-83);
// row_node maps each free block row to its mesh node, nodes are the mesh's positions.
sf_status setup_rigid_modes(cudaStream_t st, uint32_t rows, const uint32_t* row_node, const double* nodes,
                            const double center[3], double scale, double* modes);
// The coarsest level's dense Cholesky factor (in `work`, n x n) and explicit inverse L^-T L^-1 (in
// `inverse`), bit-identical to DenseCholesky's column loop (block.rs:307-374) and the host's
// inverse; `li` is n x n scratch. A non-positive pivot stops the factor: its column goes to *bad
// (which must hold ~0 before) and its value to *pivot; the inverse is then not meaningful.
sf_status setup_dense_inverse(cudaStream_t st, uint32_t rows, int rb, const uint32_t* starts, const uint32_t* cols,
                              const double* vals, size_t n, double* work, double* li, double* inverse,
                              unsigned long long* bad, double* pivot);
// The tentative prolongator of every aggregate into t (rows x rb x 6 at the members' rows) and the
// coarse near-null space (aggregates x 36), bit-identical to the host loops (transfer.rs:19-68).
// max_members: the largest aggregate's member count (its rows are staged in shared memory; an
// aggregate of more than 200 KB of rows is refused).
sf_status setup_tentative(cudaStream_t st, size_t aggregates, int rb, size_t max_members, const uint32_t* member_starts,
                          const uint32_t* members, const double* near_null, double* t, double* coarse);
sf_status setup_smooth(cudaStream_t st, int rb, size_t entries, const uint32_t* entry_row, const uint32_t* p_cols,
                       const uint32_t* a_starts, const uint32_t* a_cols, const double* a_vals, const uint32_t* n_starts,
                       const uint32_t* n_cols, const uint32_t* aggregate, const double* t_vals, const double* inv,
                       double omega, double* p_vals);
sf_status setup_product(cudaStream_t st, int rb, size_t entries, const uint32_t* entry_row, const uint32_t* ap_cols,
                        const uint32_t* a_starts, const uint32_t* a_cols, const double* a_vals, const uint32_t* p_starts,
                        const uint32_t* p_cols, const double* p_vals, double* ap_vals);
sf_status setup_galerkin(cudaStream_t st, int rb, size_t entries, const uint32_t* entry_row, const uint32_t* c_cols,
                         const uint32_t* pt_starts, const uint32_t* pt_rows, const uint32_t* pt_at, const double* p_vals,
                         const uint32_t* ap_starts, const uint32_t* ap_cols, const double* ap_vals, double* c_vals);
template <typename S>
sf_status setup_convert(cudaStream_t st, size_t n, const double* in, S* out);
template <typename S>
sf_status setup_transpose_blocks(cudaStream_t st, size_t blocks, int rb, int cb, const uint32_t* src, const double* in,
                                 S* out);
// The SELL-32 copy's columns and values (converted to S) from block CSR on the device.
template <typename S>
sf_status setup_sell_fill(cudaStream_t st, size_t slots, int len, const uint32_t* sell_rows, const uint32_t* sell_len,
                          const uint32_t* sell_start, uint32_t nrows, const uint32_t* starts, const uint32_t* cols,
                          const double* in, uint32_t* out_cols, S* out);
// The split-row copy of a 6 x cb block CSR matrix (cb 3 or 6), converted to S.
template <typename S>
sf_status setup_split_fill(cudaStream_t st, size_t slots, int cb, const uint32_t* sell_rows, const uint32_t* sell_len,
                           const uint32_t* sell_start, uint32_t nrows, const uint32_t* starts, const uint32_t* cols,
                           const double* in, uint32_t* out_cols, S* out);

// ------------------------------------------------------------------- assembly (assembly.cu)
struct AssemblyDevice {
  double* nodes = nullptr;        // node_count x 3
  uint32_t* tets = nullptr;       // tet_count x 10
  double* ke = nullptr;           // 495 x tet_count upper-triangle element stiffness
  double* point_material = nullptr;  // tet_count x points x 2 (E, nu) when a callback supplies it
  double* positions = nullptr;    // tet_count x points x 3, integration point positions
  uint32_t* inc_start = nullptr;  // node_count + 1: each node's elements in inc, ascending
  uint32_t* inc = nullptr;        // 10 x tet_count
  uint32_t* row_node = nullptr;   // per free block row: its node
  uint32_t* cursor = nullptr;     // per free block row: the next of its node's elements to add
  unsigned long long* error = nullptr;  // (tet << 32) | (point << 8) | kind, min over faults
  uint32_t tet_count = 0;
  int quadrature = 0;
  int points = 4;
};

enum { FAULT_NONE = 0, FAULT_INVERTED = 1, FAULT_MATERIAL = 2 };

// Element stiffness of elements [e0, e1) into assembly.ke (bit-exact with the reference's
// element_stiffness, crates/solidfem-elastic/src/element.rs:98-133).
sf_status launch_element_stiffness(const AssemblyDevice& a, const MaterialSpec& m, uint32_t e0,
                                   uint32_t e1, cudaStream_t stream);
// Integration point positions of all elements (for a host material callback).
sf_status launch_point_positions(const AssemblyDevice& a, cudaStream_t stream);
// Adds the stiffness of elements below `end` to the block values, each block summing its
// elements in ascending order (assembly.rs:87-130 adds them in element order).
sf_status launch_gather(const AssemblyDevice& a, DevBsr& system, uint32_t end, cudaStream_t stream);

// Device stress recovery (results.rs:470-539, patch.rs): fills point stresses, per-node worst
// values and patch fits, then the nodal field.
struct RecoveryDevice {
  double* disp = nullptr;         // node_count x 3
  uint32_t* free = nullptr;       // node_count: free index or FIXED
  double* point_stress = nullptr; // tet_count x points x 6
  double* point_vm = nullptr;     // tet_count x points
  double* point_pos = nullptr;    // tet_count x points x 3
  double* point_mat = nullptr;    // tet_count x points x 2
  double* node_candidate = nullptr;  // tet_count x 10 x 7: stress and von Mises at each node
  uint32_t* vertex_offsets = nullptr;  // vertex_count + 1
  uint32_t* vertex_incident = nullptr; // elements touching each vertex, ascending
  uint32_t* node_offsets = nullptr;    // node_count + 1: (element, local node) incidence
  uint32_t* node_incident = nullptr;   // (element << 4) | local node, ascending element
  double* fits = nullptr;         // vertex_count x 28: centre (3), scale, coefficients (4 x 6)
  int* has_fit = nullptr;         // vertex_count
  uint32_t* midside_first = nullptr;  // per midside node: (first element << 3) | edge slot
  double* nodal_stress = nullptr; // node_count x 6
  double* nodal_vm = nullptr;     // node_count
  bool ready = false;             // incidence uploaded
};
// Device stress recovery of the displacements in r.disp (crates/solidfem-elastic/src/results.rs:
// 470-539 and 376-410, patch.rs:37-120), bit-identical to the reference's serial recovery, in
// the reference's units of work: elements [first, end) (point stresses and each element's values
// at its nodes), then vertices [first, end) (patch fits), then the nodal field once both are done.
// Every unit is independent of the others, so any slicing gives the bits of one pass.
sf_status launch_recovery_elements(const AssemblyDevice& a, const MaterialSpec& m, RecoveryDevice& r, uint32_t first,
                                   uint32_t end, cudaStream_t stream);
sf_status launch_recovery_fits(const AssemblyDevice& a, RecoveryDevice& r, uint32_t first, uint32_t end,
                               cudaStream_t stream);
sf_status launch_recovery_field(const AssemblyDevice& a, RecoveryDevice& r, uint32_t node_count,
                                uint32_t vertex_count, cudaStream_t stream);
// The displacement of every mesh node from the free-DOF solution (zero at fixed nodes).
sf_status launch_scatter_displacements(const double* x, RecoveryDevice& r, uint32_t node_count, cudaStream_t stream);

// ------------------------------------------------------------------- solve (solve.cu)
// Uploads the hierarchy in the study's precision and allocates every work vector.
sf_status solver_upload_hierarchy(DeviceSolver& s, const std::vector<HostLevel>& levels,
                                  uint64_t degree);
sf_status solver_init_pcg(DeviceSolver& s, double tolerance, uint64_t max_iterations);
// Enqueues one full iteration (pcg.rs:216-275) on s.stream.
sf_status solver_enqueue_iteration(DeviceSolver& s);
// Enqueues z = M r for the current r (reset_direction, pcg.rs:278-282) and rz.
sf_status solver_enqueue_reset(DeviceSolver& s);
// One stage of a level's V-cycle (SF_STAGE_*) on f64 device buffers (inspection entry point).
sf_status solver_level_stage(DeviceSolver& s, size_t level, int stage, const double* in0, const double* in1,
                             double* out0, double* out1);
// One standalone preconditioner application / system product (inspection entry points).
sf_status solver_precondition(DeviceSolver& s, const double* d_in, double* d_out);
sf_status solver_system_multiply(DeviceSolver& s, const double* d_in, double* d_out);
sf_status solver_capture_graph(DeviceSolver& s);
sf_status solver_read_state(DeviceSolver& s, PcgState* out);
// Pcg::step on the device (study.cpp): up to max_iterations iterations replayed in chunks with one
// state read-back per chunk into `pinned`; updates last, status and cancelled.
sf_status run_iterations(DeviceSolver& d, bool use_graphs, uint64_t max_iterations, sf_cancel_fn cancel, void* user,
                         PcgState* pinned, PcgState& last, int& status, bool& cancelled);
// The step outcome of a solve in `status` and its PcgError, if it failed, as the returned status.
sf_status step_result(int status, bool cancelled, const PcgState& last, sf_step_outcome* out);
// Restarts the solve from x = 0 with the resident right-hand side (Pcg::new).
sf_status solver_restart(DeviceSolver& s, double tolerance, uint64_t max_iterations);
// Mean device milliseconds per launch of one solver kernel and its algorithmic bytes per launch.
sf_status solver_time_kernel(DeviceSolver& s, int kernel, uint64_t repeats, double* ms, double* bytes);
// Several solvers advanced together: one graph whose nodes are single grids over all of them
// (blockIdx.y = instance), each instance's arguments from a device table per launch site.
struct BatchIteration {
  cudaStream_t stream = nullptr;
  size_t count = 0, sites = 0;
  std::vector<void*> tables;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};
// Fails with SF_INVALID_ARGUMENT when the solvers do not share their launch structure.
sf_status batch_build(const std::vector<DeviceSolver*>& inst, cudaStream_t stream, BatchIteration& out);
sf_status batch_replay(BatchIteration& b, uint64_t iterations);
void batch_destroy(BatchIteration& b);

// y_k = A x_k and energy[k] = x_k . y_k for count vectors of device memory (count x n each),
// enqueued on s.stream; the reduction scratch is a static device array, so nothing is allocated.
sf_status solver_energy_products(DeviceSolver& s, const double* x, double* y, double* energy, uint64_t count);
// The most vectors one solver_energy_products call takes.
uint64_t solver_energy_max_vectors();

}  // namespace sf
