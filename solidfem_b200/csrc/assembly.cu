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

// Adds, for every block of the pattern, the contributions of its elements below `end`, resuming
// where the previous slice stopped.
__global__ void gather_kernel(size_t blocks, const uint32_t* __restrict__ map_starts, const uint32_t* __restrict__ map,
                              const double* __restrict__ ke, uint32_t* __restrict__ cursor, uint32_t end,
                              double* __restrict__ vals) {
  size_t blk = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (blk >= blocks) return;
  uint32_t j = cursor[blk], stop = map_starts[blk + 1];
  if (j == stop) return;
  double v[9];
  for (int k = 0; k < 9; ++k) v[k] = vals[blk * 9 + k];
  for (; j < stop; ++j) {
    uint32_t packed = map[j];
    uint32_t e = packed >> 7;
    if (e >= end) break;
    int ab = packed & 127, a = ab / 10, b = ab % 10;
    if (a <= b) {
      const double* src = ke + (size_t)e * 495 + (size_t)c_pair[a][b] * 9;
      for (int k = 0; k < 9; ++k) v[k] += src[k];
    } else {
      const double* src = ke + (size_t)e * 495 + (size_t)c_pair[b][a] * 9;
      for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) v[i * 3 + k] += src[k * 3 + i];
    }
  }
  cursor[blk] = j;
  for (int k = 0; k < 9; ++k) vals[blk * 9 + k] = v[k];
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
  if (system.blocks == 0) return SF_OK;
  if (sf_status s = ensure_tables(a.quadrature, stream)) return s;
  gather_kernel<<<(unsigned)((system.blocks + 255) / 256), 256, 0, stream>>>(
      system.blocks, a.map_starts, a.map, a.ke, a.cursor, end, (double*)system.vals);
  return cuda_check(cudaGetLastError(), "gather");
}

}  // namespace sf
