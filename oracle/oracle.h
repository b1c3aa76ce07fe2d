/* ORACLE — test infrastructure only: the C interface of the CPU restatement in oracle.cpp.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline load it. */
#ifndef SOLIDFEM_ORACLE_H
#define SOLIDFEM_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  ORC_OK = 0,
  ORC_MESH_EMPTY = 1,
  ORC_MESH_NONFINITE = 2,
  ORC_MESH_NODE_RANGE = 3,
  ORC_MESH_DEGENERATE = 4,
  ORC_MESH_FLAT = 5,
  ORC_MESH_UNUSED = 6,
  ORC_MESH_NONMANIFOLD = 7,
  ORC_MESH_BOX = 8,
  ORC_NO_FIXED_NODES = 20,
  ORC_BODY_NOT_HELD = 21,
  ORC_NODE_RANGE = 22,
  ORC_NONFINITE_LOAD = 23,
  ORC_FACE_NOT_ON_BOUNDARY = 24,
  ORC_NO_EFFECTIVE_LOAD = 25,
  ORC_ELEMENT_INVERTED = 26,
  ORC_ELEMENT_MATERIAL = 27,
  ORC_JACOBI_DIAGONAL = 28,
  ORC_BAD_PRESCRIBED = 31,
  ORC_MG_BLOCK_STRUCTURE = 40,
  ORC_MG_NEAR_NULL_LENGTH = 41,
  ORC_MG_NOT_POSITIVE_DEFINITE = 42,
  ORC_MG_POSITION_LENGTH = 43
};

enum { ORC_ACTIVE = 0, ORC_CONVERGED = 1, ORC_FAILED_NOT_POSITIVE_DEFINITE = 2, ORC_FAILED_NOT_CONVERGED = 3 };
enum { ORC_PRECISION_DOUBLE = 0, ORC_PRECISION_SINGLE_STORAGE = 1, ORC_PRECISION_SINGLE = 2 };
enum { ORC_PRECONDITIONER_JACOBI = 0, ORC_PRECONDITIONER_MULTIGRID = 1 };
enum { ORC_MATERIAL_UNIFORM = 0, ORC_MATERIAL_SHELL_CORE = 1 };

typedef struct {
  int32_t kind;   /* ORC_MATERIAL_* */
  double E, nu;   /* uniform material, or the shell's */
  double E2, nu2; /* the core's */
  double lo[3], hi[3];
  double depth;   /* points closer than this to a face of [lo, hi] are shell */
} orc_material;

typedef struct {
  int32_t preconditioner;
  int32_t precision;
  double tolerance;
  uint64_t max_iterations; /* 0: 10 n + 1000 */
  double neighbour_reach;
  uint64_t coarse_dofs;
  uint64_t max_levels;
  uint64_t smoother_degree;
  double smoother_range;
  int32_t quadrature; /* 0: four-point, 1: fourteen-point */
} orc_options;

typedef struct {
  uint32_t node;
  double force[3];
} orc_nodal_force;

typedef struct {
  uint32_t tet;
  uint32_t face;
  uint32_t nodes[6];
} orc_face;

typedef struct {
  uint64_t iteration;
  double relative_residual;
  int32_t at_rounding_floor;
  int32_t status;
  double fail_curvature;
} orc_progress;

typedef struct {
  uint64_t rows, row_block, blocks;
  double lambda_min, lambda_max;
  int32_t has_prolongator;
  uint64_t p_blocks, p_col_block;
  int32_t has_factor;
} orc_level_info;

typedef struct {
  uint64_t levels;
  uint64_t coarse_dofs;
  double operator_complexity;
  uint64_t memory_bytes;
} orc_mg_stats;

typedef struct {
  uint32_t tet;
  uint32_t point;
  double position[3];
  double stress[6];
  double von_mises;
} orc_point_stress;

typedef struct {
  uint32_t node;
  uint32_t axis;
  double value;
} orc_prescribed;

// Stages of one V-cycle level (orc_level_stage): smoother from zero; x + smoother; the start
// (D^-1 b) / theta; b - A x; P^T r; x + P e.
enum { ORC_STAGE_SMOOTH = 0, ORC_STAGE_RESIDUAL = 1, ORC_STAGE_RESTRICT = 2, ORC_STAGE_PROLONG = 3,
       ORC_STAGE_START = 4, ORC_STAGE_SMOOTH_ADD = 5 };
typedef struct orc_mesh orc_mesh;
typedef struct orc_study orc_study;

#ifdef __cplusplus
}
#endif
#endif
