/*
 * solidfem_b200 — C ABI of a B200-native (sm_100a) implementation of solidfem's solve path:
 * 10-node tetrahedral elasticity, device FP64 stiffness assembly, and conjugate gradients
 * preconditioned by a block smoothed-aggregation multigrid V-cycle that runs on the GPU.
 *
 * Every entry point replaces one call of the reference's Rust API (larsbrubaker/solidfem); the
 * comment above each names the reference item (path:line inside that project) whose behaviour it
 * keeps. Plain pointers and sizes only; no exceptions cross this boundary; every call returns an
 * sf_status and leaves details in a thread-local sf_error (sf_last_error).
 *
 * Ownership follows the reference: a model moves into the builder (sf_builder_create consumes
 * it, like StudyBuilder::new), a finished builder moves into the study (sf_builder_finish), and
 * results are copied into caller buffers. Handles are not thread-safe: use one per host thread.
 */
#ifndef SOLIDFEM_B200_H
#define SOLIDFEM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SF_ABI_VERSION 3

/* Status codes. Named refusals mirror MeshError (crates/solidfem-mesh/src/error.rs),
 * ModelError (crates/solidfem-elastic/src/error.rs:23-119), MultigridError
 * (crates/solidfem-solve/src/multigrid/mod.rs:199-246) and PcgError
 * (crates/solidfem-solve/src/pcg.rs:61-77). */
typedef enum sf_status {
  SF_OK = 0,
  SF_MESH_EMPTY = 1,
  SF_MESH_NON_FINITE_POSITION = 2,
  SF_MESH_NODE_OUT_OF_RANGE = 3,
  SF_MESH_DEGENERATE_TET = 4,
  SF_MESH_FLAT_TET = 5,
  SF_MESH_UNUSED_NODE = 6,
  SF_MESH_NON_MANIFOLD_FACE = 7,
  SF_MESH_INVALID_BOX = 8,
  SF_NO_FIXED_NODES = 20,
  SF_BODY_NOT_HELD = 21,
  SF_NODE_OUT_OF_RANGE = 22,
  SF_NON_FINITE_LOAD = 23,
  SF_FACE_NOT_ON_BOUNDARY = 24,
  SF_NO_EFFECTIVE_LOAD = 25,
  SF_ELEMENT_INVERTED_JACOBIAN = 26,
  SF_ELEMENT_INVALID_MATERIAL = 27,
  SF_JACOBI_DIAGONAL = 28,
  SF_CANCELLED = 29,
  SF_NOT_FINISHED = 30,
  SF_AXIS_OUT_OF_RANGE = 31,
  SF_PRESCRIBED_ON_FIXED_NODE = 32,
  SF_DOFS_DO_NOT_HOLD = 33,
  SF_MG_BLOCK_STRUCTURE = 40,
  SF_MG_NEAR_NULL_LENGTH = 41,
  SF_MG_NOT_POSITIVE_DEFINITE = 42,
  SF_MG_POSITION_LENGTH = 43,
  SF_MG_COARSEST_NOT_FACTORED = 44,
  SF_MG_COARSE_LENGTH = 45,
  SF_PCG_NOT_POSITIVE_DEFINITE = 50,
  SF_PCG_NOT_CONVERGED = 51,
  SF_INVALID_ARGUMENT = 60,
  SF_CUDA_ERROR = 61,
  SF_DEVICE_MEMORY_BUDGET = 62,
  SF_NO_DEVICE = 63,
  SF_DEVICE_WAIT_TIMEOUT = 64
} sf_status;

/* Details of the last failure on this thread: the payloads of the reference's error variants. */
typedef struct sf_error {
  int32_t status;
  uint32_t tet, node, face, point, axis;
  uint64_t row, level, block, iteration, rank;
  uint64_t expected, found; /* the lengths of NearNullLength and PositionLength */
  double pivot, curvature, relative_residual, determinant, value;
  char message[256];
} sf_error;

/* The last failure on the calling thread. */
sf_status sf_last_error(sf_error* out);
/* A static English description of a status. */
const char* sf_status_message(sf_status status);
/* SF_ABI_VERSION of the loaded library. */
int32_t sf_abi_version(void);

/* ---------------------------------------------------------------- mesh --------------------- */
typedef struct sf_mesh sf_mesh;

/* A face on the mesh boundary: BoundaryFace, crates/solidfem-mesh/src/boundary.rs:15-24. */
typedef struct sf_boundary_face {
  uint32_t tet;
  uint32_t face;     /* the corner it is opposite, 0..3 */
  uint32_t nodes[6]; /* FACE_NODES order: three corners, then edge midpoints */
} sf_boundary_face;

/* box_tet_mesh (crates/solidfem-mesh/src/box_mesh.rs:22-80) upgraded by
 * QuadraticTetMesh::from_linear (crates/solidfem-mesh/src/quadratic.rs:24-71). */
sf_status sf_box_tet_mesh(const double origin[3], const double size[3],
                          const uint64_t divisions[3], sf_mesh** out);
/* TetMesh::new (crates/solidfem-mesh/src/tet.rs:59-109) then QuadraticTetMesh::from_linear.
 * positions: n x 3, tets: ntets x 4. */
sf_status sf_mesh_from_linear(const double* positions, uint64_t n, const uint32_t* tets,
                              uint64_t ntets, sf_mesh** out);
void sf_mesh_destroy(sf_mesh* mesh);
uint64_t sf_mesh_node_count(const sf_mesh* mesh);
uint64_t sf_mesh_tet_count(const sf_mesh* mesh);
uint64_t sf_mesh_vertex_count(const sf_mesh* mesh);
/* QuadraticTetMesh::nodes / tets (quadratic.rs:74-81): node_count x 3 and tet_count x 10. */
sf_status sf_mesh_nodes(const sf_mesh* mesh, double* out);
sf_status sf_mesh_tets(const sf_mesh* mesh, uint32_t* out);
/* QuadraticTetMesh::boundary_faces (quadratic.rs:89-124), ascending by sorted corners. */
uint64_t sf_mesh_boundary_face_count(const sf_mesh* mesh);
sf_status sf_mesh_boundary_faces(const sf_mesh* mesh, sf_boundary_face* out);

/* The same meshes generated on CUDA device `device`: the nodes, ten-node tets and boundary faces
 * are those the host builders above return, bit for bit, with the same refusals (TetMesh::new's
 * checks, tet.rs:59-109). Edges and faces are bucketed by their smallest corner on the device in
 * place of the host's sorts. The mesh also keeps its ten-node arrays on that device: a study built
 * from it on the same device copies them there instead of uploading them. */
/* box_tet_mesh + QuadraticTetMesh::from_linear (box_mesh.rs:22-80, quadratic.rs:24-124). */
sf_status sf_box_tet_mesh_device(const double origin[3], const double size[3],
                                 const uint64_t divisions[3], int32_t device, sf_mesh** out);
/* TetMesh::new then QuadraticTetMesh::from_linear (tet.rs:59-109, quadratic.rs:24-124). */
sf_status sf_mesh_from_linear_device(const double* positions, uint64_t n, const uint32_t* tets,
                                     uint64_t ntets, int32_t device, sf_mesh** out);
/* The demo's part mesh, build_mesh (demo/wasm/src/part.rs:135-189) over a PartGrid: ascending grid
 * lines per axis (x_count, y_count, z_count lines), a unit box_tet_mesh of the cells, the
 * tetrahedra whose centroid's cell lies in the hollow core dropped (wall_cells > 0: cross-section
 * cells at least wall_cells in from every side, part.rs:114-122), the kept vertices numbered in
 * order of first appearance and placed on their grid lines, then TetMesh::new and from_linear. */
sf_status sf_part_tet_mesh_device(const double* x_lines, uint64_t x_count, const double* y_lines,
                                  uint64_t y_count, const double* z_lines, uint64_t z_count,
                                  uint64_t wall_cells, int32_t device, sf_mesh** out);
/* The device holding the mesh's ten-node arrays, or -1 for a mesh built on the host. */
int32_t sf_mesh_device(const sf_mesh* mesh);

/* ---------------------------------------------------------------- model -------------------- */
typedef struct sf_model sf_model;

/* Material, crates/solidfem-elastic/src/material.rs:5-31. */
typedef struct sf_material {
  double youngs_modulus;
  double poisson_ratio;
} sf_material;

/* A MaterialField (material.rs:35-50), evaluated in batches: write out[i] for positions[3i..3i+3],
 * i < count. Called on the host with the integration points' physical positions. */
typedef void (*sf_material_field_fn)(void* user, const double* positions, uint64_t count,
                                     sf_material* out);

enum { SF_QUADRATURE_FOUR_POINT = 0, SF_QUADRATURE_FOURTEEN_POINT = 1 };

/* Model::new (crates/solidfem-elastic/src/study.rs:58-68): copies the mesh. */
sf_status sf_model_create(const sf_mesh* mesh, sf_material material, sf_model** out);
void sf_model_destroy(sf_model* model);
/* A MaterialField callback in place of the uniform material. */
sf_status sf_model_set_material_field(sf_model* model, sf_material_field_fn field, void* user);
/* The printed-part field: points closer than `depth` to a face of the box [lo, hi] are `shell`,
 * the rest `core`; evaluated per integration point like any MaterialField. */
sf_status sf_model_set_shell_core(sf_model* model, sf_material shell, sf_material core,
                                  const double lo[3], const double hi[3], double depth);
/* Model::set_quadrature (study.rs:76-78). */
sf_status sf_model_set_quadrature(sf_model* model, int32_t rule);
/* Model::fix_node (study.rs:81-83); the array form fixes each listed node. */
sf_status sf_model_fix_node(sf_model* model, uint32_t node);
sf_status sf_model_fix_nodes(sf_model* model, const uint32_t* nodes, uint64_t count);
/* Model::add_nodal_force (study.rs:86-88). */
sf_status sf_model_add_nodal_force(sf_model* model, uint32_t node, const double force[3]);
/* Model::add_traction (study.rs:101-103); the array form adds count faces, tractions count x 3. */
sf_status sf_model_add_traction(sf_model* model, const sf_boundary_face* face,
                                const double traction[3]);
sf_status sf_model_add_tractions(sf_model* model, const sf_boundary_face* faces,
                                 const double* tractions, uint64_t count);
/* Model::prescribe_displacement (study.rs:96-98). */
sf_status sf_model_prescribe_displacement(sf_model* model, uint32_t node, uint32_t axis,
                                          double value);

/* ---------------------------------------------------------------- options ------------------ */
enum { SF_PRECONDITIONER_JACOBI = 0, SF_PRECONDITIONER_MULTIGRID = 1 };
/* Precision (crates/solidfem-solve/src/multigrid/mod.rs:127-141) plus MIXED: the Single cycle
 * (f32 storage and vectors) inside an FP64 flexible conjugate gradient. */
enum {
  SF_PRECISION_DOUBLE = 0,
  SF_PRECISION_SINGLE_STORAGE = 1,
  SF_PRECISION_SINGLE = 2,
  SF_PRECISION_MIXED = 3
};

/* StudyOptions (study.rs:139-148) with PcgOptions (pcg.rs:14-33) and MultigridOptions
 * (multigrid/mod.rs:143-182), plus device settings. */
typedef struct sf_study_options {
  double tolerance;        /* 1e-9 */
  uint64_t max_iterations; /* 0: 10 n + 1000 */
  int32_t preconditioner;  /* SF_PRECONDITIONER_* ; the reference's default is Jacobi */
  double neighbour_reach;  /* 3.0 */
  uint64_t coarse_dofs;    /* 1500 */
  uint64_t max_levels;     /* 12 */
  uint64_t smoother_degree;/* 3 */
  double smoother_range;   /* 30.0 */
  int32_t precision;       /* SF_PRECISION_* ; SINGLE_STORAGE */
  uint64_t threads;        /* host threads for setup; 0: half the logical processors, at most 8 */
  int32_t device;          /* CUDA device ordinal */
  int32_t use_graphs;      /* capture each solver iteration in a CUDA graph (default 1) */
  uint64_t device_memory_budget; /* bytes a study may hold on the device; 0: no limit */
  uint64_t sell_min_rows;  /* operators with at least this many block rows use the SELL-32 layout;
                              0: 32768 */
  int32_t batchable;       /* lay every operator out by its block shape alone (no SELL, fixed lanes
                              per row), so studies of the same depth can share a batch
                              (sf_study_solve_batch); default 0 */
  int32_t coarse_tail;     /* run the last smoothed level and the coarse direct solve as one
                              thread-block-cluster launch when they are small enough (same results,
                              bit for bit, as the per-phase launches); default 0: on the 606k-DOF
                              plate the cluster launch takes 44 us against about 37 us for the
                              per-phase launches it replaces. Not used by batchable studies. */
} sf_study_options;

/* StudyOptions::default with the reference's defaults (Jacobi preconditioner). */
void sf_study_options_default(sf_study_options* options);

/* Returns nonzero to cancel. Read before each slice of assembly, each phase of each multigrid
 * setup level, each solver iteration and each recovery launch (the reference reads it per element,
 * per setup row and per iteration; the device does those in larger launches). */
typedef int32_t (*sf_cancel_fn)(void* user);

/* ---------------------------------------------------------------- build -------------------- */
typedef struct sf_builder sf_builder;
typedef struct sf_study sf_study;

/* BuildProgress, study.rs:381-390. */
typedef struct sf_build_progress {
  uint64_t elements_done;
  uint64_t elements_total;
  int32_t setup_finished;
} sf_build_progress;

/* StudyBuilder::new (study.rs:419-474): validates, builds the load and the pattern. Consumes
 * `model` whatever the outcome. */
sf_status sf_builder_create(sf_model* model, const sf_study_options* options, sf_builder** out);
/* StudyBuilder::step (study.rs:478-512): adds the stiffness of up to max_elements more elements
 * (on the device), then advances the multigrid setup by up to max_elements block rows. Any
 * slicing gives the bits of one call. */
sf_status sf_builder_step(sf_builder* builder, uint64_t max_elements, sf_cancel_fn cancel,
                          void* user, sf_build_progress* progress);
/* StudyBuilder::finish (study.rs:601-656): on success consumes the builder. */
sf_status sf_builder_finish(sf_builder* builder, sf_study** out);
void sf_builder_destroy(sf_builder* builder);
/* StaticStudy::new (study.rs:191-199): create + step(all) + finish. Consumes `model`. */
sf_status sf_study_create(sf_model* model, const sf_study_options* options, sf_cancel_fn cancel,
                          void* user, sf_study** out);

/* ---------------------------------------------------------------- solve -------------------- */
/* Progress, pcg.rs:36-45. */
typedef struct sf_progress {
  uint64_t iteration;
  double relative_residual;
  int32_t at_rounding_floor;
} sf_progress;

/* StepOutcome, pcg.rs:47-57. */
enum { SF_OUTCOME_RUNNING = 0, SF_OUTCOME_CONVERGED = 1, SF_OUTCOME_CANCELLED = 2 };
typedef struct sf_step_outcome {
  int32_t kind;
  sf_progress progress;
} sf_step_outcome;

/* StaticStudy::step (study.rs:202-215): up to max_iterations device iterations; the same bits
 * however the solve is sliced. */
sf_status sf_study_step(sf_study* study, uint64_t max_iterations, sf_cancel_fn cancel, void* user,
                        sf_step_outcome* outcome);
/* Pcg::progress (pcg.rs:200-207) of the study's solve: iterations, relative residual, floor. */
sf_status sf_study_progress(const sf_study* study, sf_progress* out);
/* StaticStudy::displacements (study.rs:219-238): node_count x 3, zero at fixed nodes. The estimate
 * so far (Pcg::estimate, pcg.rs:192-194) while the solve runs: a preview, not an answer. */
sf_status sf_study_displacements(const sf_study* study, double* out);

/* Report, study.rs:151-176. */
typedef struct sf_report {
  uint64_t total_dofs;
  uint64_t free_dofs;
  uint64_t nonzeros;
  int32_t at_rounding_floor;
  uint64_t iterations;
  double relative_residual;
  double assembly_seconds;
  double preconditioner_seconds;
  double solve_seconds;
  double recovery_seconds;
  int32_t has_multigrid;
  uint64_t mg_levels;
  uint64_t mg_coarse_dofs;
  double mg_operator_complexity;
  uint64_t mg_memory_bytes;
} sf_report;
sf_status sf_study_report(const sf_study* study, sf_report* out);

/* PointStress, crates/solidfem-elastic/src/results.rs:66-79. */
typedef struct sf_point_stress {
  uint32_t tet;
  uint32_t point;
  double position[3];
  double stress[6];
  double von_mises;
} sf_point_stress;

/* StaticStudy::solution (study.rs:246-260), recovered on the device: refuses with
 * SF_NOT_FINISHED before convergence. `cancel` is read between slices of 65,536 units of recovery
 * work (SF_CANCELLED); the recovered field is kept, so later calls only copy it out. Any output
 * pointer may be NULL. displacements: node_count x 3; nodal_stress: node_count x 6;
 * nodal_von_mises: node_count; points: tet_count x points_per_element. */
sf_status sf_study_solution(sf_study* study, sf_cancel_fn cancel, void* user, double* displacements,
                            double* nodal_stress, double* nodal_von_mises, sf_point_stress* points);

/* Recovery (crates/solidfem-elastic/src/results.rs:97-124): a resumable stress recovery of one
 * snapshot of a study's displacements, with its own device buffers. Its study may be destroyed
 * first: the recovery's device memory then goes with the study, and the handle only accepts
 * sf_recovery_destroy. */
typedef struct sf_recovery sf_recovery;
/* StaticStudy::begin_recovery (study.rs:262-274): snapshots the current displacements on the
 * device: the converged answer, or a preview of a solve still running. */
sf_status sf_study_begin_recovery(sf_study* study, sf_recovery** out);
/* StaticStudy::continue_recovery (study.rs:276-296): up to max_units more units of work (each
 * element, then each vertex's patch fit, in order, on the device); *finished (may be NULL) is
 * set once all are done. `cancel` is read before each launch (SF_CANCELLED; the recovery can be
 * continued later). Any slicing gives the bits of one call. An inverted element or invalid
 * material is refused by name (tet, point). */
sf_status sf_study_continue_recovery(sf_study* study, sf_recovery* recovery, uint64_t max_units,
                                     sf_cancel_fn cancel, void* user, int32_t* finished);
/* StaticStudy::finish_recovery (study.rs:298-304): the recovered field (RecoveredField,
 * results.rs:126-139), outputs as sf_study_solution; SF_NOT_FINISHED while units remain. */
sf_status sf_study_finish_recovery(sf_study* study, sf_recovery* recovery, double* displacements,
                                   double* nodal_stress, double* nodal_von_mises, sf_point_stress* points);
void sf_recovery_destroy(sf_recovery* recovery);
void sf_study_destroy(sf_study* study);

/* ------------------------------------------------------------- raw systems ---------------- */
/* The solver crate's seam without a mesh: a symmetric matrix in scalar CSR (CsrMatrix,
 * crates/solidfem-solve/src/csr.rs:6-13) and a right-hand side, solved on the device by the
 * conjugate gradient of Pcg::new / step / estimate / progress (pcg.rs:133-213). options->
 * preconditioner picks Jacobi::new (preconditioner.rs:49-79) or the multigrid of
 * MultigridSetup::new + step + finish (multigrid/setup.rs:129-215, run to the end inside create,
 * `cancel` read before each phase of each level); the other options are the study's (tolerance, cap, multigrid
 * settings, precision, device, graphs). */
typedef struct sf_system sf_system;

/* n unknowns; row_starts n + 1, columns and values row_starts[n] each (every row's columns
 * strictly ascending and below n: SF_INVALID_ARGUMENT otherwise); rhs n. For multigrid,
 * near_null holds near_null_count = 6 n values ((row, mode) at 6 row + mode) and positions
 * position_count = n / 3 points (x, y, z), one per block row; wrong lengths are refused as
 * SF_MG_NEAR_NULL_LENGTH / SF_MG_POSITION_LENGTH (expected, found in sf_error), a matrix whose
 * rows do not group into 3x3 blocks as SF_MG_BLOCK_STRUCTURE (row), a diagonal block that is not
 * positive definite as SF_MG_NOT_POSITIVE_DEFINITE (level, block, pivot). For Jacobi they are
 * ignored, n is any size, and a diagonal entry that is not positive and finite is refused as
 * SF_JACOBI_DIAGONAL (row, value). options NULL: the defaults (Jacobi). A zero right-hand side
 * is converged at once. */
sf_status sf_system_create(uint64_t n, const uint64_t* row_starts, const uint32_t* columns, const double* values,
                           const double* rhs, const double* near_null, uint64_t near_null_count,
                           const double* positions, uint64_t position_count, const sf_study_options* options,
                           sf_cancel_fn cancel, void* user, sf_system** out);
/* Pcg::step (pcg.rs:167-190): up to max_iterations iterations, the same bits however sliced;
 * SF_PCG_NOT_POSITIVE_DEFINITE (iteration, curvature) or SF_PCG_NOT_CONVERGED (iteration,
 * relative_residual) once the solve has failed, for this call and every later one. */
sf_status sf_system_step(sf_system* system, uint64_t max_iterations, sf_cancel_fn cancel, void* user,
                         sf_step_outcome* outcome);
/* Pcg::estimate (pcg.rs:192-194): the current estimate, n values. */
sf_status sf_system_estimate(const sf_system* system, double* out);
/* Pcg::progress (pcg.rs:200-207). */
sf_status sf_system_progress(const sf_system* system, sf_progress* out);
/* Multigrid::level_sizes().len() (cycle.rs:333-339); 0 under Jacobi. */
uint64_t sf_system_level_count(const sf_system* system);
void sf_system_destroy(sf_system* system);

/* ------------------------------------------------------------- inspection ----------------- */
/* The assembled free-DOF system as scalar CSR (csr.rs:6-13), copied from the device:
 * row_starts free_dofs + 1, columns and values nonzeros each. */
sf_status sf_study_matrix(const sf_study* study, uint64_t* row_starts, uint32_t* columns,
                          double* values);
/* The right-hand side over the free DOFs (study.rs:444-449). */
sf_status sf_study_rhs(const sf_study* study, double* out);

/* Multigrid::level_sizes (cycle.rs:333-339) and MultigridStats (mod.rs:186-195). */
uint64_t sf_study_level_count(const sf_study* study);
typedef struct sf_level_info {
  uint64_t rows, row_block, blocks;
  double lambda_min, lambda_max;
  int32_t has_prolongator;
  uint64_t prolongator_blocks;
  int32_t has_factor;
} sf_level_info;
sf_status sf_study_level_info(const sf_study* study, uint64_t level, sf_level_info* out);
/* Multigrid::level_matrix / level_prolongator (cycle.rs:367-385): the level's f64 setup values
 * (before any rounding to the stored precision). starts rows + 1, columns blocks. */
sf_status sf_study_level_matrix(const sf_study* study, uint64_t level, int32_t prolongator,
                                uint64_t* starts, uint32_t* columns, double* values);
/* Multigrid::aggregates (cycle.rs:355-361): one per block row, empty on the coarsest level. */
sf_status sf_study_aggregates(const sf_study* study, uint64_t level, uint32_t* out);
/* Preconditioner::apply (preconditioner.rs:10-20): one device V-cycle (or Jacobi scaling) of
 * `residual` into `output`, free_dofs each, host buffers. */
sf_status sf_study_precondition(sf_study* study, const double* residual, double* output);
/* The stages of one level of the device V-cycle (cycle.rs:461-539 and its device form,
 * gpu/reference.rs:17-240), each run by exactly the launches the cycle makes for it, in the
 * study's storage and vector precision (host f64 buffers; inputs are rounded to the vector type,
 * outputs widened): the hand-off the reference's device tests compare stage by stage
 * (tests/solver/gpu_hierarchy_execution.rs:434-557). n is the level's scalar rows, nc the next
 * coarser level's.
 *   SMOOTH          in0 b (n) -> out0 the smoother from zero (n)
 *   SMOOTH_ADD      in0 b, in1 x (n) -> out0 x + smoother (the post-smoother's final add)
 *   START           in0 b (n) -> out0 (D^-1 b) / theta (the smoother's first iterate)
 *   RESIDUAL        in0 b, in1 x (n) -> out0 b - A x
 *   RESTRICT        in0 r (n) -> out0 R r (nc)
 *   PROLONG         in0 e (nc), in1 x (n) -> out0 x + P e
 *   RESTRICT_START  in0 r (n) -> out0 R r (nc), out1 the coarser level's start from it (nc)
 *   RESIDUAL_START  in0 b, in1 x (n) -> out0 b - A x, out1 the start from it (n)
 * The stage overwrites the level's work vectors: call it between solver steps, not during one. */
enum {
  SF_STAGE_SMOOTH = 0,
  SF_STAGE_RESIDUAL = 1,
  SF_STAGE_RESTRICT = 2,
  SF_STAGE_PROLONG = 3,
  SF_STAGE_START = 4,
  SF_STAGE_SMOOTH_ADD = 5,
  SF_STAGE_RESTRICT_START = 6,
  SF_STAGE_RESIDUAL_START = 7
};
sf_status sf_study_level_stage(sf_study* study, uint64_t level, int32_t stage, const double* in0,
                               const double* in1, double* out0, double* out1);
/* CsrMatrix::multiply (csr.rs:112-120) on the device, FP64, host buffers. */
sf_status sf_study_system_multiply(sf_study* study, const double* x, double* y);

/* No counterpart in the reference. System products with their energies, on device memory the
 * caller owns, allocating nothing: for k < count, y_k = A x_k and energy[k] = x_k . y_k in FP64,
 * where x_k and y_k are the free-DOF vectors at x + k * free_dofs and y + k * free_dofs.
 *
 * For callers that must not allocate device memory on this path: a serving loop that has given
 * its whole device budget to resident studies, or one that keeps other streams busy, where
 * cudaMalloc can fail and cudaFree waits for the whole device. (sf_study_system_multiply
 * allocates two device buffers per call and copies through the host.) The reduction's scratch is
 * a static 65,792-byte device array in this library, one per device.
 *
 * - count at most 8; a larger count is refused with SF_INVALID_ARGUMENT before any work. count 0
 *   does nothing. x, y and energy: 8-byte-aligned device (or managed) memory of the study's
 *   device, not overlapping; x and y hold count * free_dofs doubles, energy count doubles, each
 *   range inside one allocation (a range that runs past the end of its allocation is refused;
 *   the driver sees allocations only, so a sub-allocator's piece is checked against the whole
 *   allocation it was carved from).
 * - The calling thread's current device is the same after the call as before it.
 * - Asynchronous: the kernel is enqueued on the study's stream (sf_study_stream); read y and
 *   energy after that stream has reached it.
 * - The first call on a device looks up the scratch's address with that device current, which can
 *   load this library's device code on it. Make that first call before any stream capture begins
 *   on the device.
 * - The scratch holds arrival tickets that must be zero when a call starts: they are zero when the
 *   library loads, and each call leaves them at zero when its kernel completes. Nothing else in
 *   it needs an initial value.
 * - Every study on a device shares the one scratch array: two calls whose kernels can run at the
 *   same time (different streams, studies or host threads) race and give wrong results. Order
 *   them, for example on one stream.
 * - The scratch's address is kept per device for the life of the process. Studies and this address
 *   do not survive cudaDeviceReset: destroy every study of a device before resetting it, and do not
 *   call this entry point on that device afterwards. */
sf_status sf_study_energy_products(sf_study* study, const double* x, double* y, double* energy,
                                   uint64_t count);

/* ------------------------------------------------------------- re-solve and timing -------- */
/* Restarts the solve from a zero estimate (Pcg::new, pcg.rs:135-164) on the resident matrix and
 * preconditioner, with a new right-hand side over the free DOFs (host buffer), or the resident
 * one when `rhs` is NULL. The reference builds a new Pcg for a new load; this keeps the assembled
 * system and hierarchy on the device. */
sf_status sf_study_resolve(sf_study* study, const double* rhs);

/* No counterpart in the reference: batched solves. Restarts every listed study from a zero
 * estimate on its resident right-hand side and solves them together: each kernel of a conjugate
 * gradient step is ONE grid over all of them (blockIdx.y selects the study, whose operator,
 * vectors and scalars come from a per-study argument table), and each study's own status word
 * masks its blocks once it has converged or failed. Runs until every study has stopped; studies
 * that stopped leave the batch between chunks of iterations. The studies must share their device
 * and their launch structure (the same number of levels and the same operator layouts, as small
 * studies of the same depth do); SF_INVALID_ARGUMENT otherwise. outcomes and statuses (either may
 * be NULL) receive count entries: each study's outcome and its SF_OK / SF_PCG_NOT_CONVERGED /
 * SF_PCG_NOT_POSITIVE_DEFINITE. */
sf_status sf_study_solve_batch(sf_study** studies, uint64_t count, sf_step_outcome* outcomes,
                               sf_status* statuses);

/* The CUDA stream (cudaStream_t as an integer) every kernel of the study is launched on, so a
 * caller can bracket work with its own CUDA events. */
uint64_t sf_study_stream(const sf_study* study);

/* Device time of the last sf_study_step call (CUDA events on the study's stream), the device time
 * of the assembly, the kernels launched so far and the bytes copied each way. */
typedef struct sf_device_timing {
  double step_ms;
  double assembly_ms;
  double setup_ms;
  uint64_t kernel_launches;
  uint64_t h2d_bytes;
  uint64_t d2h_bytes;
  uint64_t launches_per_iteration; /* kernels one conjugate gradient iteration launches */
  int32_t coarse_tail_level;       /* the level whose cycle runs as one cluster launch, or -1 */
  uint32_t coarse_tail_cluster;    /* CTAs of that cluster (0 without a coarse tail) */
} sf_device_timing;
sf_status sf_study_device_timing(const sf_study* study, sf_device_timing* out);

/* Times one solver kernel in isolation: `repeats` launches between CUDA events on the study's
 * stream. kernel: SF_KERNEL_*. Returns the mean milliseconds per launch and the kernel's
 * algorithmic bytes per launch (every value, index and vector entry it must move once). */
enum {
  SF_KERNEL_CHEBYSHEV_STEP = 0, /* finest level: A d, r -= A d, z = D^-1 r, d, x updates */
  SF_KERNEL_LEVEL_RESIDUAL = 1, /* finest level: r = b - A x in the cycle's precision */
  SF_KERNEL_SYSTEM_PRODUCT = 2, /* the FP64 system product of the conjugate gradient */
  SF_KERNEL_RESTRICTION = 3     /* finest level: P^T r through the stored transpose */
};
typedef struct sf_kernel_timing {
  double ms_per_launch;
  double bytes_per_launch;
  uint64_t launches;
} sf_kernel_timing;
sf_status sf_study_time_kernel(sf_study* study, int32_t kernel, uint64_t repeats, sf_kernel_timing* out);

/* ------------------------------------------------------------- serving ------------------- */
/* No counterpart in the reference: a request loop for many solves on one GPU. Requests are
 * admitted in arrival order while their device memory fits `memory_budget`, built on host worker
 * threads (each study on its own CUDA stream, hierarchy and vectors resident on the device) and
 * solved. Studies with fewer than `batch_max_dofs` free DOFs are built batchable and solved in
 * continuous batches: between chunks of iterations a batch drops the studies that stopped and
 * takes in the ones that became ready, and each step is one grid per kernel over all its studies
 * (sf_study_solve_batch). Larger studies solve on their own streams from solver threads,
 * overlapping on the device with the batches and with each other. */
typedef struct sf_server sf_server;
typedef struct sf_server_options {
  int32_t device;
  uint64_t memory_budget;  /* bytes of device memory for admitted requests; 0: 150 GiB */
  uint64_t batch_max_dofs; /* requests with fewer free DOFs are batched; 100000 by default */
  uint64_t max_batch;      /* studies per batch; 0: 64 */
  uint64_t build_threads;  /* host threads building requests; 0: 8 */
  uint64_t solve_threads;  /* host threads driving the solves too large to batch; 0: 4 */
  uint64_t setup_threads;  /* host threads inside one build when its options leave it 0; 0: 2 */
} sf_server_options;
void sf_server_options_default(sf_server_options* options);
sf_status sf_server_create(const sf_server_options* options, sf_server** out);
/* Submits a model (consumed) with its study options; `id` names the request. */
sf_status sf_server_submit(sf_server* server, sf_model* model, const sf_study_options* options,
                           uint64_t* id);

typedef struct sf_request_result {
  int32_t status;    /* the request's sf_status once finished */
  int32_t finished;
  int32_t batched;
  uint64_t batch_size; /* the largest batch it ran in */
  sf_step_outcome outcome;
  uint64_t free_dofs, node_count, device_bytes;
  double queue_seconds, build_seconds, solve_seconds, latency_seconds; /* latency from submission */
  char message[160]; /* the failure's sf_error message, empty on success */
} sf_request_result;
/* Waits up to timeout_ms (UINT64_MAX: until done) for a request; SF_NOT_FINISHED while it runs. */
sf_status sf_server_wait(sf_server* server, uint64_t id, uint64_t timeout_ms, sf_request_result* out);
/* Copies a finished request's displacements (node_count x 3, may be NULL) and forgets the request;
 * returns the request's own failure status if it failed. */
sf_status sf_server_take(sf_server* server, uint64_t id, double* displacements);

/* Cancels a request: one still queued is dropped at once; one being built or solved stops at its
 * next cancel check (a batched one leaves its batch between chunks of iterations, the other
 * members going on). It then finishes with status SF_CANCELLED. A finished request is left as it
 * is. */
sf_status sf_server_cancel(sf_server* server, uint64_t id);

typedef struct sf_server_stats {
  uint64_t completed, pending, reserved_bytes, peak_reserved_bytes, batches, batched_requests;
  double mean_batch_size; /* studies per batched chunk */
} sf_server_stats;
sf_status sf_server_statistics(sf_server* server, sf_server_stats* out);
/* Stops taking requests, finishes the builds and batches in flight, then frees everything;
 * requests not yet admitted are dropped. */
void sf_server_destroy(sf_server* server);

#ifdef __cplusplus
}
#endif
#endif
