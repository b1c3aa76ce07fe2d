// FP64 stiffness assembly on sm_100a, bit-identical to the reference's serial assembly. This file
// is built with -fmad=false (no fused multiply-add, which the reference never uses) and IEEE
// division and square root, and every sum runs in the reference's order:
//  * element_stiffness_kernel: one thread per element integrates the 30x30 B^T D B
//    (crates/solidfem-elastic/src/element.rs:98-133). Only the 55 blocks a <= b are stored: the
//    reference writes each lower block as the mirror of the same value, so they are equal bits.
//  * gather_kernel: one thread per 3x3 block of the free-node pattern adds its elements'
//    contributions in ascending element order, which is the order the reference's element loop
//    adds them in (crates/solidfem-elastic/src/assembly.rs:87-130).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>

#include "device.h"

namespace sf {

namespace {

struct QuadratureTable {
  double der[14][10][3];
  double val[14][10];
  double weight[14];
};
__constant__ QuadratureTable c_rule;
__constant__ int c_pair[10][10];  // index of block (a, b), a <= b, among the 55 stored

struct FieldArgs {
  int kind;
  double E, nu, E2, nu2;
  double lo[3], hi[3];
  double depth;
};

// The MaterialField at a position: uniform, or the shell/core part (points nearer than `depth` to
// a face of [lo, hi] are shell).
__device__ __forceinline__ void field_at(const FieldArgs& f, const double* p, double& E, double& nu) {
  if (f.kind == MATERIAL_SHELL_CORE) {
    double depth = INFINITY;
    for (int a = 0; a < 3; ++a) {
      depth = fmin(depth, p[a] - f.lo[a]);
      depth = fmin(depth, f.hi[a] - p[a]);
    }
    if (depth < f.depth) {
      E = f.E;
      nu = f.nu;
    } else {
      E = f.E2;
      nu = f.nu2;
    }
  } else {
    E = f.E;
    nu = f.nu;
  }
}

// point_geometry (element.rs:25-80) at rule point q; returns the determinant and fills the
// gradients and the position.
__device__ __forceinline__ double geometry(const double (&x)[10][3], int q, double (&g)[10][3], double (&pos)[3]) {
  double j[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  pos[0] = pos[1] = pos[2] = 0.0;
  for (int a = 0; a < 10; ++a)
    for (int i = 0; i < 3; ++i) {
      for (int k = 0; k < 3; ++k) j[i][k] += c_rule.der[q][a][i] * x[a][k];
      pos[i] += c_rule.val[q][a] * x[a][i];
    }
  double cof[3][3];
  cof[0][0] = j[1][1] * j[2][2] - j[1][2] * j[2][1];
  cof[0][1] = j[0][2] * j[2][1] - j[0][1] * j[2][2];
  cof[0][2] = j[0][1] * j[1][2] - j[0][2] * j[1][1];
  cof[1][0] = j[1][2] * j[2][0] - j[1][0] * j[2][2];
  cof[1][1] = j[0][0] * j[2][2] - j[0][2] * j[2][0];
  cof[1][2] = j[0][2] * j[1][0] - j[0][0] * j[1][2];
  cof[2][0] = j[1][0] * j[2][1] - j[1][1] * j[2][0];
  cof[2][1] = j[0][1] * j[2][0] - j[0][0] * j[2][1];
  cof[2][2] = j[0][0] * j[1][1] - j[0][1] * j[1][0];
  double det = j[0][0] * cof[0][0] + j[0][1] * cof[1][0] + j[0][2] * cof[2][0];
  for (int a = 0; a < 10; ++a)
    for (int k = 0; k < 3; ++k) {
      double sum = cof[k][0] * c_rule.der[q][a][0] + cof[k][1] * c_rule.der[q][a][1] + cof[k][2] * c_rule.der[q][a][2];
      g[a][k] = sum / det;
    }
  return det;
}

// Shared-memory slots per thread and integration point: 30 gradients, lambda, mu, measure.
const int kSlots = 33;

__global__ void element_stiffness_kernel(const double* __restrict__ nodes, const uint32_t* __restrict__ tets,
                                         uint32_t e0, uint32_t e1, int points, FieldArgs field,
                                         const double* __restrict__ point_material, double* __restrict__ ke,
                                         unsigned long long* error) {
  extern __shared__ double sm[];
  uint32_t e = e0 + blockIdx.x * blockDim.x + threadIdx.x;
  int t = threadIdx.x, nt = blockDim.x;
  bool live = e < e1;
  bool ok = live;
  if (live) {
    double x[10][3];
    for (int a = 0; a < 10; ++a) {
      uint32_t n = tets[(size_t)e * 10 + a];
      for (int k = 0; k < 3; ++k) x[a][k] = nodes[(size_t)n * 3 + k];
    }
    for (int q = 0; q < points && ok; ++q) {
      double g[10][3], pos[3];
      double det = geometry(x, q, g, pos);
      if (isnan(det) || det <= 0.0) {
        atomicMin(error, ((unsigned long long)e << 32) | ((unsigned long long)q << 8) | FAULT_INVERTED);
        ok = false;
        break;
      }
      double E, nu;
      if (point_material) {
        E = point_material[((size_t)e * points + q) * 2];
        nu = point_material[((size_t)e * points + q) * 2 + 1];
      } else {
        field_at(field, pos, E, nu);
      }
      bool valid = isfinite(E) && E > 0.0 && nu > -1.0 && nu < 0.5;
      if (!valid) {
        atomicMin(error, ((unsigned long long)e << 32) | ((unsigned long long)q << 8) | FAULT_MATERIAL);
        ok = false;
        break;
      }
      // Material::lame, material.rs:24-31.
      double lambda = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
      double mu = E / (2.0 * (1.0 + nu));
      double measure = c_rule.weight[q] * det / 6.0;
      double* slot = sm + (size_t)q * kSlots * nt + t;
      for (int a = 0; a < 10; ++a)
        for (int k = 0; k < 3; ++k) slot[(a * 3 + k) * nt] = g[a][k];
      slot[30 * nt] = lambda;
      slot[31 * nt] = mu;
      slot[32 * nt] = measure;
    }
  }
  if (!ok) return;
  double* out = ke + (size_t)e * 495;
  for (int a = 0; a < 10; ++a)
    for (int b = a; b < 10; ++b) {
      double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int q = 0; q < points; ++q) {
        const double* slot = sm + (size_t)q * kSlots * nt + t;
        double ga[3], gb[3];
        for (int k = 0; k < 3; ++k) {
          ga[k] = slot[(a * 3 + k) * nt];
          gb[k] = slot[(b * 3 + k) * nt];
        }
        double lambda = slot[30 * nt], mu = slot[31 * nt], measure = slot[32 * nt];
        double dot = ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2];
        for (int i = 0; i < 3; ++i)
          for (int k = 0; k < 3; ++k) {
            double value = lambda * (ga[i] * gb[k]) + mu * (ga[k] * gb[i]);
            if (i == k) value += mu * dot;
            value *= measure;
            acc[i * 3 + k] += value;
          }
      }
      double* o = out + (size_t)c_pair[a][b] * 9;
      for (int v = 0; v < 9; ++v) o[v] = acc[v];
    }
}

// Integration point positions, for a material callback evaluated on the host.
__global__ void point_positions_kernel(const double* __restrict__ nodes, const uint32_t* __restrict__ tets,
                                       uint32_t count, int points, double* __restrict__ positions) {
  uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= count) return;
  double x[10][3];
  for (int a = 0; a < 10; ++a) {
    uint32_t n = tets[(size_t)e * 10 + a];
    for (int k = 0; k < 3; ++k) x[a][k] = nodes[(size_t)n * 3 + k];
  }
  for (int q = 0; q < points; ++q) {
    double pos[3] = {0, 0, 0};
    for (int a = 0; a < 10; ++a)
      for (int i = 0; i < 3; ++i) pos[i] += c_rule.val[q][a] * x[a][i];
    for (int i = 0; i < 3; ++i) positions[((size_t)e * points + q) * 3 + i] = pos[i];
  }
}

// Adds to every block of the pattern the contributions of its elements below `end`, resuming
// where the previous slice stopped: one warp per block row (free node). The warp stages up to 32
// of the node's elements (ascending, from the row's cursor) with their ten nodes and the node's
// place in each; lane j then walks them in order for block j of the row and, where an element
// also holds the block's column node, adds that element's (a, b) block. Each block therefore
// sums its elements in ascending order, the order of the reference's element loop
// (assembly.rs:87-130); no per-block list of contributions exists. A row sums only its blocks on
// and above the diagonal and writes each off-diagonal one's mirror (column, row) as its
// transpose: an element's (b, a) block is the transpose of its (a, b) block to the bit (the
// reference mirrors the value), so the mirror's sum over the same elements in the same order is
// that transpose, and every element block is read once.
constexpr int kGatherWarps = 8;
constexpr int kGatherStage = 32;

__global__ void __launch_bounds__(32 * kGatherWarps)
    gather_kernel(uint32_t rows, const uint32_t* __restrict__ starts, const uint32_t* __restrict__ cols,
                  const uint32_t* __restrict__ row_node, const uint32_t* __restrict__ inc_start,
                  const uint32_t* __restrict__ inc, const uint32_t* __restrict__ tets,
                  const double* __restrict__ ke, uint32_t* __restrict__ cursor, uint32_t end,
                  double* __restrict__ vals) {
  __shared__ uint32_t s_nodes[kGatherWarps][kGatherStage][10];
  __shared__ uint32_t s_elem[kGatherWarps][kGatherStage];
  __shared__ int s_place[kGatherWarps][kGatherStage];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned full = 0xffffffffu;
  for (uint32_t r = blockIdx.x * kGatherWarps + warp; r < rows; r += gridDim.x * kGatherWarps) {
    const uint32_t node = row_node[r], k0 = cursor[r], k1 = inc_start[node + 1];
    const uint32_t b0 = starts[r], nb = starts[r + 1] - b0;
    // the row's first block on or above the diagonal (columns ascend)
    uint32_t lo = 0, hi = nb;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (cols[b0 + mid] < r)
        lo = mid + 1;
      else
        hi = mid;
    }
    const uint32_t upper = lo;
    uint32_t k_end = k0;
    for (uint32_t jb = upper; jb < nb; jb += 32) {
      const uint32_t j = jb + lane;
      const bool live = j < nb;
      const uint32_t col_node = live ? row_node[cols[b0 + j]] : 0xffffffffu;
      // a row's first slice starts its blocks from zero (the values were zeroed at allocation)
      // without reading them; later slices resume from the stored sums
      const bool resume = k0 != inc_start[node];
      double v[9];
#pragma unroll
      for (int q = 0; q < 9; ++q) v[q] = live && resume ? vals[(size_t)(b0 + j) * 9 + q] : 0.0;
      uint32_t k = k0;
      for (;;) {
        // stage the next elements below `end` (they are ascending: the first at or past `end`
        // ends the row's work for this slice)
        const uint32_t kk = k + lane;
        const uint32_t e = kk < k1 ? inc[kk] : 0xffffffffu;
        const bool take = kk < k1 && e < end;
        const unsigned mask = __ballot_sync(full, take);
        const int count = __popc(mask);  // a prefix: elements ascend
        if (take) {
          s_elem[warp][lane] = e;
          int place = 0;
#pragma unroll
          for (int q = 0; q < 10; ++q) {
            const uint32_t n = tets[(size_t)e * 10 + q];
            s_nodes[warp][lane][q] = n;
            if (n == node) place = q;
          }
          s_place[warp][lane] = place;
        }
        __syncwarp();
        if (live) {
          for (int t = 0; t < count; ++t) {
            int b = -1;
#pragma unroll
            for (int q = 0; q < 10; ++q)
              if (s_nodes[warp][t][q] == col_node) b = q;
            if (b < 0) continue;
            const int a = s_place[warp][t];
            const size_t el = s_elem[warp][t];
            if (a <= b) {
              const double* src = ke + el * 495 + (size_t)c_pair[a][b] * 9;
#pragma unroll
              for (int q = 0; q < 9; ++q) v[q] += src[q];
            } else {
              const double* src = ke + el * 495 + (size_t)c_pair[b][a] * 9;
#pragma unroll
              for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int q = 0; q < 3; ++q) v[i * 3 + q] += src[q * 3 + i];
            }
          }
        }
        __syncwarp();
        k += (uint32_t)count;
        if (count < 32) break;
      }
      k_end = k;
      if (live) {
#pragma unroll
        for (int q = 0; q < 9; ++q) vals[(size_t)(b0 + j) * 9 + q] = v[q];
        const uint32_t col = cols[b0 + j];
        if (col != r) {
          // the mirror block (col, r) in row col: the transpose
          uint32_t mlo = starts[col], mhi = starts[col + 1];
          while (mlo < mhi) {
            const uint32_t mid = (mlo + mhi) >> 1;
            if (cols[mid] < r)
              mlo = mid + 1;
            else
              mhi = mid;
          }
          if (mlo < starts[col + 1] && cols[mlo] == r)
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
              for (int q = 0; q < 3; ++q) vals[(size_t)mlo * 9 + q * 3 + i] = v[i * 3 + q];
        }
      }
    }
    if (lane == 0) cursor[r] = k_end;
  }
}

// The rules' points (crates/solidfem-elastic/src/quadrature.rs:111-144) and the Tet10 shape
// functions at them (crates/solidfem-elastic/src/shape.rs:25-67), evaluated once on the host in
// the reference's operation order (the host build does not contract multiplies and adds).
QuadratureTable make_table(int quadrature) {
  static const double A4 = 0.1381966011250105, B4 = 0.5854101966249685;
  static const double A14 = 0.3108859192633006, W14A = 0.11268792571801585;
  static const double C14 = 0.09273525031089123, W14B = 0.07349304311636195;
  static const double E14 = 0.04550370412564965, W14C = 0.042546020777081466;
  const double B14 = 1.0 - 3.0 * A14, D14 = 1.0 - 3.0 * C14, F14 = 0.5 - E14;
  const double four[4][4] = {{A4, A4, A4, 0.25}, {B4, A4, A4, 0.25}, {A4, B4, A4, 0.25}, {A4, A4, B4, 0.25}};
  const double fourteen[14][4] = {
      {A14, A14, A14, W14A}, {B14, A14, A14, W14A}, {A14, B14, A14, W14A}, {A14, A14, B14, W14A},
      {C14, C14, C14, W14B}, {D14, C14, C14, W14B}, {C14, D14, C14, W14B}, {C14, C14, D14, W14B},
      {E14, E14, F14, W14C}, {E14, F14, E14, W14C}, {F14, E14, E14, W14C}, {E14, F14, F14, W14C},
      {F14, E14, F14, W14C}, {F14, F14, E14, W14C}};
  static const int edges[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
  static const double dl[4][3] = {{-1.0, -1.0, -1.0}, {1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
  QuadratureTable t;
  std::memset(&t, 0, sizeof(t));
  int count = quadrature == SF_QUADRATURE_FOURTEEN_POINT ? 14 : 4;
  for (int q = 0; q < count; ++q) {
    const double* p = quadrature == SF_QUADRATURE_FOURTEEN_POINT ? fourteen[q] : four[q];
    double r = p[0], s = p[1], u = p[2];
    double l[4];
    l[0] = 1.0 - r - s - u;
    l[1] = r;
    l[2] = s;
    l[3] = u;
    for (int i = 0; i < 4; ++i) t.val[q][i] = l[i] * (2.0 * l[i] - 1.0);
    for (int e = 0; e < 6; ++e) t.val[q][4 + e] = 4.0 * l[edges[e][0]] * l[edges[e][1]];
    for (int axis = 0; axis < 3; ++axis) {
      for (int i = 0; i < 4; ++i) t.der[q][i][axis] = (4.0 * l[i] - 1.0) * dl[i][axis];
      for (int e = 0; e < 6; ++e) {
        int a = edges[e][0], b = edges[e][1];
        t.der[q][4 + e][axis] = 4.0 * (dl[a][axis] * l[b] + l[a] * dl[b][axis]);
      }
    }
    t.weight[q] = p[3];
  }
  return t;
}

int g_table_rule = -1;

sf_status ensure_tables(int quadrature, cudaStream_t stream) {
  if (g_table_rule == quadrature) return SF_OK;
  QuadratureTable t = make_table(quadrature);
  int pair[10][10];
  int k = 0;
  for (int a = 0; a < 10; ++a)
    for (int b = 0; b < 10; ++b) pair[a][b] = -1;
  for (int a = 0; a < 10; ++a)
    for (int b = a; b < 10; ++b) pair[a][b] = k++;
  cudaError_t e = cudaMemcpyToSymbolAsync(c_rule, &t, sizeof(t), 0, cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) e = cudaMemcpyToSymbolAsync(c_pair, pair, sizeof(pair), 0, cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return cuda_check(e, "quadrature tables");
  g_table_rule = quadrature;
  return SF_OK;
}

FieldArgs field_args(const MaterialSpec& m) {
  FieldArgs f;
  std::memset(&f, 0, sizeof(f));
  f.kind = m.kind;
  if (m.kind == MATERIAL_SHELL_CORE) {
    f.E = m.shell.youngs_modulus;
    f.nu = m.shell.poisson_ratio;
    f.E2 = m.core.youngs_modulus;
    f.nu2 = m.core.poisson_ratio;
    for (int a = 0; a < 3; ++a) {
      f.lo[a] = m.lo[a];
      f.hi[a] = m.hi[a];
    }
    f.depth = m.depth;
  } else {
    f.E = m.uniform.youngs_modulus;
    f.nu = m.uniform.poisson_ratio;
  }
  return f;
}

}  // namespace

sf_status launch_element_stiffness(const AssemblyDevice& a, const MaterialSpec& m, uint32_t e0, uint32_t e1,
                                   cudaStream_t stream) {
  if (e1 <= e0) return SF_OK;
  if (sf_status s = ensure_tables(a.quadrature, stream)) return s;
  int threads = a.points > 4 ? 32 : 64;
  size_t smem = (size_t)a.points * kSlots * threads * sizeof(double);
  cudaFuncSetAttribute(element_stiffness_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  uint32_t count = e1 - e0;
  element_stiffness_kernel<<<(count + threads - 1) / threads, threads, smem, stream>>>(
      a.nodes, a.tets, e0, e1, a.points, field_args(m), a.point_material, a.ke, a.error);
  return cuda_check(cudaGetLastError(), "element stiffness");
}

sf_status launch_point_positions(const AssemblyDevice& a, cudaStream_t stream) {
  if (sf_status s = ensure_tables(a.quadrature, stream)) return s;
  point_positions_kernel<<<(a.tet_count + 127) / 128, 128, 0, stream>>>(a.nodes, a.tets, a.tet_count, a.points,
                                                                         a.positions);
  return cuda_check(cudaGetLastError(), "point positions");
}

sf_status launch_gather(const AssemblyDevice& a, DevBsr& system, uint32_t end, cudaStream_t stream) {
  if (system.blocks == 0 || system.rows == 0) return SF_OK;
  if (sf_status s = ensure_tables(a.quadrature, stream)) return s;
  const unsigned grid = (unsigned)std::min<size_t>((system.rows + kGatherWarps - 1) / kGatherWarps, 148 * 64);
  gather_kernel<<<grid, 32 * kGatherWarps, 0, stream>>>(system.rows, system.starts, system.cols, a.row_node,
                                                        a.inc_start, a.inc, a.tets, a.ke, a.cursor, end,
                                                        (double*)system.vals);
  return cuda_check(cudaGetLastError(), "gather");
}


// ============================================================ stress recovery
// crates/solidfem-elastic/src/results.rs:470-539 (elements, then vertex patch fits) and 376-410
// (the nodal field), crates/solidfem-elastic/src/patch.rs:37-120, one thread per element, vertex
// or node, every sum in the reference's order.

namespace {

struct NodeTable {
  double der[10][10][3];  // shape derivatives at each element node's natural coordinates
  int nearest[10];        // the integration point nearest each node (results.rs:555-569)
};
__constant__ NodeTable c_node;
int g_node_rule = -1;

void shape_derivatives_host(const double nat[3], double d[10][3]) {
  static const int edges[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
  static const double dl[4][3] = {{-1.0, -1.0, -1.0}, {1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
  double l[4] = {1.0 - nat[0] - nat[1] - nat[2], nat[0], nat[1], nat[2]};
  for (int axis = 0; axis < 3; ++axis) {
    for (int i = 0; i < 4; ++i) d[i][axis] = (4.0 * l[i] - 1.0) * dl[i][axis];
    for (int e = 0; e < 6; ++e) {
      int a = edges[e][0], b = edges[e][1];
      d[4 + e][axis] = 4.0 * (dl[a][axis] * l[b] + l[a] * dl[b][axis]);
    }
  }
}

sf_status ensure_node_table(int quadrature, cudaStream_t stream) {
  if (g_node_rule == quadrature) return SF_OK;
  static const double natural[10][3] = {{0, 0, 0},     {1, 0, 0},     {0, 1, 0},   {0, 0, 1},
                                        {0.5, 0, 0},   {0.5, 0.5, 0}, {0, 0.5, 0}, {0, 0, 0.5},
                                        {0.5, 0, 0.5}, {0, 0.5, 0.5}};
  NodeTable t;
  for (int n = 0; n < 10; ++n) shape_derivatives_host(natural[n], t.der[n]);
  // The rule's points, as make_table lists them.
  QuadratureTable rule = make_table(quadrature);
  (void)rule;
  static const double A4 = 0.1381966011250105, B4 = 0.5854101966249685;
  static const double A14 = 0.3108859192633006, C14 = 0.09273525031089123, E14 = 0.04550370412564965;
  const double B14 = 1.0 - 3.0 * A14, D14 = 1.0 - 3.0 * C14, F14 = 0.5 - E14;
  const double four[4][3] = {{A4, A4, A4}, {B4, A4, A4}, {A4, B4, A4}, {A4, A4, B4}};
  const double fourteen[14][3] = {{A14, A14, A14}, {B14, A14, A14}, {A14, B14, A14}, {A14, A14, B14},
                                  {C14, C14, C14}, {D14, C14, C14}, {C14, D14, C14}, {C14, C14, D14},
                                  {E14, E14, F14}, {E14, F14, E14}, {F14, E14, E14}, {E14, F14, F14},
                                  {F14, E14, F14}, {F14, F14, E14}};
  int count = quadrature == SF_QUADRATURE_FOURTEEN_POINT ? 14 : 4;
  for (int n = 0; n < 10; ++n) {
    double best = 1.7976931348623157e308;
    int index = 0;
    for (int q = 0; q < count; ++q) {
      const double* p = quadrature == SF_QUADRATURE_FOURTEEN_POINT ? fourteen[q] : four[q];
      double d = 0.0;
      for (int a = 0; a < 3; ++a) d = d + (p[a] - natural[n][a]) * (p[a] - natural[n][a]);
      if (d < best) {
        best = d;
        index = q;
      }
    }
    t.nearest[n] = index;
  }
  cudaError_t e = cudaMemcpyToSymbolAsync(c_node, &t, sizeof(t), 0, cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return cuda_check(e, "node tables");
  g_node_rule = quadrature;
  return SF_OK;
}

// point_geometry at element node n (gradients only; element.rs:25-80).
__device__ __forceinline__ double node_geometry(const double (&x)[10][3], int n, double (&g)[10][3]) {
  double j[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int a = 0; a < 10; ++a)
    for (int i = 0; i < 3; ++i)
      for (int k = 0; k < 3; ++k) j[i][k] += c_node.der[n][a][i] * x[a][k];
  double cof[3][3];
  cof[0][0] = j[1][1] * j[2][2] - j[1][2] * j[2][1];
  cof[0][1] = j[0][2] * j[2][1] - j[0][1] * j[2][2];
  cof[0][2] = j[0][1] * j[1][2] - j[0][2] * j[1][1];
  cof[1][0] = j[1][2] * j[2][0] - j[1][0] * j[2][2];
  cof[1][1] = j[0][0] * j[2][2] - j[0][2] * j[2][0];
  cof[1][2] = j[0][2] * j[1][0] - j[0][0] * j[1][2];
  cof[2][0] = j[1][0] * j[2][1] - j[1][1] * j[2][0];
  cof[2][1] = j[0][1] * j[2][0] - j[0][0] * j[2][1];
  cof[2][2] = j[0][0] * j[1][1] - j[0][1] * j[1][0];
  double det = j[0][0] * cof[0][0] + j[0][1] * cof[1][0] + j[0][2] * cof[2][0];
  for (int a = 0; a < 10; ++a)
    for (int k = 0; k < 3; ++k) {
      double sum = cof[k][0] * c_node.der[n][a][0] + cof[k][1] * c_node.der[n][a][1] + cof[k][2] * c_node.der[n][a][2];
      g[a][k] = sum / det;
    }
  return det;
}

// strain_at then stress_at then von_mises (element.rs:159-189).
__device__ __forceinline__ double stress_of(const double (&g)[10][3], const double (&u)[10][3], double E, double nu,
                                            double (&s)[6]) {
  double h[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int a = 0; a < 10; ++a)
    for (int i = 0; i < 3; ++i)
      for (int k = 0; k < 3; ++k) h[i][k] += u[a][i] * g[a][k];
  double e[6] = {h[0][0], h[1][1], h[2][2], h[0][1] + h[1][0], h[1][2] + h[2][1], h[2][0] + h[0][2]};
  double lambda = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
  double mu = E / (2.0 * (1.0 + nu));
  double trace = e[0] + e[1] + e[2];
  s[0] = lambda * trace + 2.0 * mu * e[0];
  s[1] = lambda * trace + 2.0 * mu * e[1];
  s[2] = lambda * trace + 2.0 * mu * e[2];
  s[3] = mu * e[3];
  s[4] = mu * e[4];
  s[5] = mu * e[5];
  double a0 = s[0] - s[1], b0 = s[1] - s[2], c0 = s[2] - s[0];
  return sqrt(0.5 * (a0 * a0 + b0 * b0 + c0 * c0) + 3.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]));
}

// Per element: stress at every integration point, and at every element node with the element's own
// material (results.rs:494-523).
__global__ void recover_elements_kernel(const double* __restrict__ nodes, const uint32_t* __restrict__ tets,
                                        const double* __restrict__ disp, uint32_t first, uint32_t count, int points,
                                        FieldArgs field,
                                        const double* __restrict__ point_material, double* __restrict__ pstress,
                                        double* __restrict__ pvm, double* __restrict__ ppos, double* __restrict__ pmat,
                                        double* __restrict__ cand, unsigned long long* error) {
  uint32_t e = first + blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= count) return;
  double x[10][3], u[10][3];
  for (int a = 0; a < 10; ++a) {
    uint32_t n = tets[(size_t)e * 10 + a];
    for (int k = 0; k < 3; ++k) {
      x[a][k] = nodes[(size_t)n * 3 + k];
      u[a][k] = disp[(size_t)n * 3 + k];
    }
  }
  for (int q = 0; q < points; ++q) {
    double g[10][3], pos[3];
    double det = geometry(x, q, g, pos);
    if (isnan(det) || det <= 0.0) {
      atomicMin(error, ((unsigned long long)e << 32) | ((unsigned long long)q << 8) | FAULT_INVERTED);
      return;
    }
    double E, nu;
    if (point_material) {
      E = point_material[((size_t)e * points + q) * 2];
      nu = point_material[((size_t)e * points + q) * 2 + 1];
    } else {
      field_at(field, pos, E, nu);
    }
    if (!(isfinite(E) && E > 0.0 && nu > -1.0 && nu < 0.5)) {
      atomicMin(error, ((unsigned long long)e << 32) | ((unsigned long long)q << 8) | FAULT_MATERIAL);
      return;
    }
    double s6[6];
    double vm = stress_of(g, u, E, nu, s6);
    size_t pq = (size_t)e * points + q;
    for (int k = 0; k < 6; ++k) pstress[pq * 6 + k] = s6[k];
    pvm[pq] = vm;
    for (int k = 0; k < 3; ++k) ppos[pq * 3 + k] = pos[k];
    pmat[pq * 2] = E;
    pmat[pq * 2 + 1] = nu;
  }
  for (int n = 0; n < 10; ++n) {
    double g[10][3];
    double det = node_geometry(x, n, g);
    if (isnan(det) || det <= 0.0) {
      atomicMin(error, ((unsigned long long)e << 32) | (1ull << 16) | ((unsigned long long)n << 8) | FAULT_INVERTED);
      return;
    }
    size_t pq = (size_t)e * points + c_node.nearest[n];
    double s6[6];
    double vm = stress_of(g, u, pmat[pq * 2], pmat[pq * 2 + 1], s6);
    double* c = cand + ((size_t)e * 10 + n) * 7;
    for (int k = 0; k < 6; ++k) c[k] = s6[k];
    c[6] = vm;
  }
}

// Gaussian elimination with partial pivoting on the 4 x 4 normal equations (patch.rs:83-120).
__device__ bool patch_solve(double (&m)[4][4], double (&rhs)[4][6]) {
  for (int c = 0; c < 4; ++c) {
    int pivot = c;
    for (int r = c + 1; r < 4; ++r)
      if (fabs(m[r][c]) > fabs(m[pivot][c])) pivot = r;
    if (fabs(m[pivot][c]) <= 1e-12) return false;
    for (int k = 0; k < 4; ++k) {
      double t = m[c][k];
      m[c][k] = m[pivot][k];
      m[pivot][k] = t;
    }
    for (int k = 0; k < 6; ++k) {
      double t = rhs[c][k];
      rhs[c][k] = rhs[pivot][k];
      rhs[pivot][k] = t;
    }
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

// The linear patch fit at every mesh vertex over its elements' integration points, in element
// order; a patch of more than one material is left unfitted (results.rs:438-466, patch.rs:37-66).
__global__ void patch_fit_kernel(const double* __restrict__ nodes, uint32_t first, uint32_t vertices, int points,
                                 const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ incident,
                                 const double* __restrict__ pstress, const double* __restrict__ ppos,
                                 const double* __restrict__ pmat, double* __restrict__ fits, int* __restrict__ has_fit) {
  uint32_t v = first + blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= vertices) return;
  double c[3] = {nodes[(size_t)v * 3], nodes[(size_t)v * 3 + 1], nodes[(size_t)v * 3 + 2]};
  uint32_t o0 = offsets[v], o1 = offsets[v + 1];
  bool uniform = true;
  double E0 = 0, nu0 = 0;
  double scale = 0.0;
  bool any = false;
  for (uint32_t k = o0; k < o1; ++k) {
    size_t base = (size_t)incident[k] * points;
    for (int q = 0; q < points; ++q) {
      size_t pq = base + q;
      double E = pmat[pq * 2], nu = pmat[pq * 2 + 1];
      if (!any) {
        E0 = E;
        nu0 = nu;
        any = true;
      } else if (__double_as_longlong(E) != __double_as_longlong(E0) || __double_as_longlong(nu) != __double_as_longlong(nu0)) {
        uniform = false;
      }
      for (int a = 0; a < 3; ++a) scale = fmax(scale, fabs(ppos[pq * 3 + a] - c[a]));
    }
  }
  has_fit[v] = 0;
  if (!uniform || !any || scale == 0.0) return;
  double m[4][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}};
  double rhs[4][6];
  for (int i = 0; i < 4; ++i)
    for (int k = 0; k < 6; ++k) rhs[i][k] = 0.0;
  for (uint32_t k = o0; k < o1; ++k) {
    size_t base = (size_t)incident[k] * points;
    for (int q = 0; q < points; ++q) {
      size_t pq = base + q;
      double t[4] = {1.0, (ppos[pq * 3] - c[0]) / scale, (ppos[pq * 3 + 1] - c[1]) / scale, (ppos[pq * 3 + 2] - c[2]) / scale};
      for (int i = 0; i < 4; ++i) {
        for (int j = 0; j < 4; ++j) m[i][j] += t[i] * t[j];
        for (int comp = 0; comp < 6; ++comp) rhs[i][comp] += t[i] * pstress[pq * 6 + comp];
      }
    }
  }
  if (!patch_solve(m, rhs)) return;
  double* f = fits + (size_t)v * 28;
  f[0] = c[0];
  f[1] = c[1];
  f[2] = c[2];
  f[3] = scale;
  for (int i = 0; i < 4; ++i)
    for (int k = 0; k < 6; ++k) f[4 + i * 6 + k] = rhs[i][k];
  has_fit[v] = 1;
}

// PatchFit::at (patch.rs:69-78).
__device__ __forceinline__ void fit_at(const double* __restrict__ f, const double* p, double (&out)[6]) {
  double t[4] = {1.0, (p[0] - f[0]) / f[3], (p[1] - f[1]) / f[3], (p[2] - f[2]) / f[3]};
  for (int k = 0; k < 6; ++k) out[k] = 0.0;
  for (int term = 0; term < 4; ++term)
    for (int k = 0; k < 6; ++k) out[k] += t[term] * f[4 + term * 6 + k];
}

// The recovered nodal field (results.rs:376-410): a vertex reads its fit (or its worst incident
// element value), a midside the mean of its edge's two vertex fits at its own position.
__global__ void nodal_field_kernel(const double* __restrict__ nodes, const uint32_t* __restrict__ tets, uint32_t count,
                                   uint32_t vertices, const uint32_t* __restrict__ node_offsets,
                                   const uint32_t* __restrict__ node_incident, const double* __restrict__ cand,
                                   const double* __restrict__ fits, const int* __restrict__ has_fit,
                                   const uint32_t* __restrict__ midside_first, double* __restrict__ out6,
                                   double* __restrict__ vm) {
  uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= count) return;
  static const int edges[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
  double s[6];
  // Worst incident element value at the node: the first strictly largest in element order.
  double worst[6] = {0, 0, 0, 0, 0, 0}, best = -1.7976931348623157e308;
  for (uint32_t k = node_offsets[n]; k < node_offsets[n + 1]; ++k) {
    uint32_t inc = node_incident[k];
    const double* c = cand + ((size_t)(inc >> 4) * 10 + (inc & 15u)) * 7;
    if (c[6] > best) {
      best = c[6];
      for (int i = 0; i < 6; ++i) worst[i] = c[i];
    }
  }
  const double* p = nodes + (size_t)n * 3;
  bool done = false;
  if (n < vertices) {
    if (has_fit[n]) {
      fit_at(fits + (size_t)n * 28, p, s);
      done = true;
    }
  } else {
    uint32_t first = midside_first[n - vertices];
    uint32_t e = first >> 3, slot = first & 7u;
    uint32_t a = tets[(size_t)e * 10 + edges[slot][0]], b = tets[(size_t)e * 10 + edges[slot][1]];
    if (has_fit[a] && has_fit[b]) {
      double pa[6], pb[6];
      fit_at(fits + (size_t)a * 28, p, pa);
      fit_at(fits + (size_t)b * 28, p, pb);
      for (int k = 0; k < 6; ++k) s[k] = 0.5 * (pa[k] + pb[k]);
      done = true;
    }
  }
  if (!done)
    for (int k = 0; k < 6; ++k) s[k] = worst[k];
  for (int k = 0; k < 6; ++k) out6[(size_t)n * 6 + k] = s[k];
  double a0 = s[0] - s[1], b0 = s[1] - s[2], c0 = s[2] - s[0];
  vm[n] = sqrt(0.5 * (a0 * a0 + b0 * b0 + c0 * c0) + 3.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]));
}

__global__ void scatter_displacements_kernel(const double* __restrict__ x, const uint32_t* __restrict__ free,
                                             uint32_t count, double* __restrict__ disp) {
  uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= count) return;
  uint32_t f = free[n];
  for (int k = 0; k < 3; ++k) disp[(size_t)n * 3 + k] = f == 0xffffffffu ? 0.0 : x[(size_t)f * 3 + k];
}

}  // namespace

sf_status launch_scatter_displacements(const double* x, RecoveryDevice& r, uint32_t node_count, cudaStream_t stream) {
  scatter_displacements_kernel<<<(node_count + 255) / 256, 256, 0, stream>>>(x, r.free, node_count, r.disp);
  return cuda_check(cudaGetLastError(), "scatter displacements");
}

sf_status launch_recovery_elements(const AssemblyDevice& a, const MaterialSpec& m, RecoveryDevice& r, uint32_t first,
                                   uint32_t end, cudaStream_t stream) {
  if (end <= first) return SF_OK;
  if (sf_status s = ensure_tables(a.quadrature, stream)) return s;
  if (sf_status s = ensure_node_table(a.quadrature, stream)) return s;
  recover_elements_kernel<<<(end - first + 127) / 128, 128, 0, stream>>>(
      a.nodes, a.tets, r.disp, first, end, a.points, field_args(m), a.point_material, r.point_stress, r.point_vm,
      r.point_pos, r.point_mat, r.node_candidate, a.error);
  return cuda_check(cudaGetLastError(), "recovery elements");
}

sf_status launch_recovery_fits(const AssemblyDevice& a, RecoveryDevice& r, uint32_t first, uint32_t end,
                               cudaStream_t stream) {
  if (end <= first) return SF_OK;
  patch_fit_kernel<<<(end - first + 127) / 128, 128, 0, stream>>>(a.nodes, first, end, a.points, r.vertex_offsets,
                                                                  r.vertex_incident, r.point_stress, r.point_pos,
                                                                  r.point_mat, r.fits, r.has_fit);
  return cuda_check(cudaGetLastError(), "recovery patch fits");
}

sf_status launch_recovery_field(const AssemblyDevice& a, RecoveryDevice& r, uint32_t node_count,
                                uint32_t vertex_count, cudaStream_t stream) {
  nodal_field_kernel<<<(node_count + 127) / 128, 128, 0, stream>>>(a.nodes, a.tets, node_count, vertex_count,
                                                                   r.node_offsets, r.node_incident, r.node_candidate,
                                                                   r.fits, r.has_fit, r.midside_first, r.nodal_stress,
                                                                   r.nodal_vm);
  return cuda_check(cudaGetLastError(), "recovery field");
}

}  // namespace sf
