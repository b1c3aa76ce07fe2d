// Tet10 mesh generation on the device: the structured box (crates/solidfem-mesh/src/box_mesh.rs:
// 22-80), the demo's graded part grid with a hollow core (demo/wasm/src/part.rs:135-189), the
// checks of TetMesh::new (tet.rs:59-109), the ten-node upgrade (quadratic.rs:24-71) and the
// boundary faces (quadratic.rs:89-124). The result is the mesh the host builders make, bit for
// bit: the same node coordinates, the same midside numbering (unique edges in sorted order), the
// same boundary faces in the same order. Compiled without multiply-add contraction, so every
// coordinate is the reference's own rounding.
//
// Sorting is replaced by bucketing on the smallest corner: an edge (a < b) lands in a's bucket
// and a face with sorted corners (k0 < k1 < k2) in k0's; a thread sorts its bucket (a few dozen
// entries) and the buckets follow node order, so walking them bucket by bucket IS the sorted
// order of the keys. Offsets come from exclusive scans of the bucket counts.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>

#include "sf_internal.h"
#include "device.h"

namespace sf {

namespace {

constexpr int kT = 256;

__constant__ int kdFace[4][6] = {{1, 2, 3, 5, 9, 8}, {0, 3, 2, 7, 9, 6}, {0, 1, 3, 4, 8, 7}, {0, 2, 1, 6, 5, 4}};
__constant__ int kdEdge[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
__constant__ int kdOrder[6][3] = {{0, 1, 2}, {1, 2, 0}, {2, 0, 1}, {0, 2, 1}, {2, 1, 0}, {1, 0, 2}};

unsigned grid_of(size_t n) {
  size_t b = (n + kT - 1) / kT;
  return (unsigned)std::max<size_t>(1, std::min<size_t>(b, 148 * 32));
}

#define GRID_STRIDE(i, n) for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (n); i += (size_t)gridDim.x * blockDim.x)

// ------------------------------------------------------------------ exclusive scan of u32 counts
// out[i] = in[0] + ... + in[i - 1] for i <= n (out[n] is the total). Blocks of 1024 scan their
// slice, one block scans the slice totals, and the totals are added back.
__device__ __forceinline__ uint32_t block_inclusive_scan(uint32_t v, uint32_t* warp_tot) {
  const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (unsigned)o) x += y;
  }
  if (lane == 31) warp_tot[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = warp_tot[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= (unsigned)o) w += y;
    }
    warp_tot[lane] = w;
  }
  __syncthreads();
  const uint32_t r = x + (warp > 0 ? warp_tot[warp - 1] : 0u);
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(1024) scan_blocks_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                           uint32_t* __restrict__ sums, size_t n) {
  __shared__ uint32_t warp_tot[32];
  const size_t i = blockIdx.x * 1024ull + threadIdx.x;
  const uint32_t v = i < n ? in[i] : 0u;
  const uint32_t inc = block_inclusive_scan(v, warp_tot);
  if (i < n) out[i] = inc - v;
  if (threadIdx.x == 1023) sums[blockIdx.x] = inc;
}

__global__ void __launch_bounds__(1024) scan_sums_kernel(uint32_t* __restrict__ sums, size_t nb, uint32_t* __restrict__ total) {
  __shared__ uint32_t warp_tot[32];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (size_t c = 0; c < nb; c += 1024) {
    const size_t i = c + threadIdx.x;
    const uint32_t v = i < nb ? sums[i] : 0u;
    const uint32_t inc = block_inclusive_scan(v, warp_tot);
    const uint32_t base = carry;
    if (i < nb) sums[i] = base + inc - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry = base + inc;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void scan_add_kernel(uint32_t* __restrict__ out, const uint32_t* __restrict__ sums, size_t n) {
  GRID_STRIDE(i, n) out[i] += sums[i / 1024];
}

// ------------------------------------------------------------------ the box and the part grid
__device__ __forceinline__ double box_coord(double o, double s, uint64_t i, uint64_t d) {
  return i == d ? o + s : o + s * ((double)i / (double)d);
}

struct Box {
  double o[3], s[3];
  uint64_t d[3];
};

__global__ void box_vertices_kernel(Box b, double* __restrict__ pos, size_t n) {
  const uint64_t n0 = b.d[0] + 1, n1 = b.d[1] + 1;
  GRID_STRIDE(v, n) {
    const uint64_t at[3] = {v % n0, (v / n0) % n1, v / (n0 * n1)};
#pragma unroll
    for (int a = 0; a < 3; ++a) pos[3 * v + a] = box_coord(b.o[a], b.s[a], at[a], b.d[a]);
  }
}

// Six tets per cell around the body diagonal (box_mesh.rs:53-78): cell-major, orientation minor.
__device__ __forceinline__ void box_tet(const Box& b, size_t t, uint32_t (&v)[4]) {
  const uint64_t n0 = b.d[0] + 1, n1 = b.d[1] + 1;
  const size_t cell = t / 6;
  const int o = (int)(t % 6);
  uint64_t at[3] = {cell % b.d[0], (cell / b.d[0]) % b.d[1], cell / (b.d[0] * b.d[1])};
  uint32_t w[4];
  w[0] = (uint32_t)(at[0] + n0 * (at[1] + n1 * at[2]));
  for (int s = 0; s < 3; ++s) {
    at[kdOrder[o][s]] += 1;
    w[s + 1] = (uint32_t)(at[0] + n0 * (at[1] + n1 * at[2]));
  }
  v[0] = w[0];
  v[3] = w[3];
  if (o < 3) {
    v[1] = w[1];
    v[2] = w[2];
  } else {
    v[1] = w[2];
    v[2] = w[1];
  }
}

__global__ void box_tets_kernel(Box b, uint32_t* __restrict__ tets, size_t ntets) {
  GRID_STRIDE(t, ntets) {
    uint32_t v[4];
    box_tet(b, t, v);
#pragma unroll
    for (int c = 0; c < 4; ++c) tets[4 * t + c] = v[c];
  }
}

// part.rs:135-160: a unit tet is kept unless the cell of its centroid (the floor of the centroid's
// unit-grid coordinates, summed as sum + p * 0.25 from zero) lies in the hollow.
struct PartCells {
  uint64_t ny, nz, wall;
};
__device__ __forceinline__ bool part_hollow(const PartCells& g, uint64_t j, uint64_t k) {
  return g.wall > 0 && j >= g.wall && j < g.ny - g.wall && k >= g.wall && k < g.nz - g.wall;
}

__global__ void part_keep_kernel(Box unit, PartCells g, const double* __restrict__ pos, uint32_t* __restrict__ keep,
                                 size_t ntets) {
  GRID_STRIDE(t, ntets) {
    uint32_t v[4];
    box_tet(unit, t, v);
    double c[3] = {0.0, 0.0, 0.0};
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int a = 0; a < 3; ++a) c[a] = c[a] + pos[3 * (size_t)v[q] + a] * 0.25;
    keep[t] = part_hollow(g, (uint64_t)floor(c[1]), (uint64_t)floor(c[2])) ? 0u : 1u;
  }
}

// The kept tets in unit order, and for each unit vertex the first (kept tet, corner) naming it:
// part.rs numbers vertices in that order of first appearance.
__global__ void part_compact_kernel(Box unit, const uint32_t* __restrict__ keep, const uint32_t* __restrict__ at,
                                    uint32_t* __restrict__ kept, unsigned int* __restrict__ first, size_t ntets) {
  GRID_STRIDE(t, ntets) {
    if (!keep[t]) continue;
    uint32_t v[4];
    box_tet(unit, t, v);
    const uint32_t k = at[t];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      kept[4 * (size_t)k + c] = v[c];
      atomicMin(first + v[c], 4u * k + (uint32_t)c);
    }
  }
}

__global__ void part_mark_kernel(const unsigned int* __restrict__ first, uint32_t* __restrict__ mark, size_t nverts) {
  GRID_STRIDE(v, nverts) if (first[v] != 0xffffffffu) mark[first[v]] = 1u;
}

__global__ void part_positions_kernel(Box unit, const unsigned int* __restrict__ first, const uint32_t* __restrict__ rank,
                                      const double* __restrict__ xl, const double* __restrict__ yl,
                                      const double* __restrict__ zl, double* __restrict__ pos, size_t nverts) {
  const uint64_t n0 = unit.d[0] + 1, n1 = unit.d[1] + 1;
  GRID_STRIDE(v, nverts) {
    if (first[v] == 0xffffffffu) continue;
    const uint64_t at[3] = {v % n0, (v / n0) % n1, v / (n0 * n1)};
    const uint32_t r = rank[first[v]];
    // the unit grid's coordinate, rounded back to its grid line (part.rs:168-172)
    const double* lines[3] = {xl, yl, zl};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double p = box_coord(unit.o[a], unit.s[a], at[a], unit.d[a]);
      pos[3 * (size_t)r + a] = lines[a][(size_t)round(p)];
    }
  }
}

__global__ void part_remap_kernel(const unsigned int* __restrict__ first, const uint32_t* __restrict__ rank,
                                  uint32_t* __restrict__ tets, size_t n) {
  GRID_STRIDE(i, n) tets[i] = rank[first[tets[i]]];
}

// ------------------------------------------------------------------ TetMesh::new's checks
__device__ __forceinline__ double tet_volume(const double* a, const double* b, const double* c, const double* d) {
  double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  double v[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  double w[3] = {d[0] - a[0], d[1] - a[1], d[2] - a[2]};
  double det = u[0] * (v[1] * w[2] - v[2] * w[1]) - u[1] * (v[0] * w[2] - v[2] * w[0]) +
               u[2] * (v[0] * w[1] - v[1] * w[0]);
  return det / 6.0;
}

__device__ __forceinline__ double length2(const double* p, const double* q) {
  return (p[0] - q[0]) * (p[0] - q[0]) + (p[1] - q[1]) * (p[1] - q[1]) + (p[2] - q[2]) * (p[2] - q[2]);
}

__device__ __forceinline__ double relative_volume(const double* a, const double* b, const double* c, const double* d,
                                                  double volume) {
  const double ls[6] = {length2(a, b), length2(a, c), length2(a, d), length2(b, c), length2(b, d), length2(c, d)};
  double longest = 0.0;
  for (int i = 0; i < 6; ++i) longest = longest < ls[i] ? ls[i] : longest;
  return 6.0 * volume / (longest * sqrt(longest));
}

struct Checks {
  unsigned int nonfinite_node;  // first node with a non-finite coordinate
  unsigned int bad_tet;         // first tetrahedron that fails a check
  unsigned int unused_node;     // first node no tetrahedron names
  unsigned int non_manifold;    // nonzero when a face has three or more tetrahedra
  // the first bad tetrahedron's failure, in TetMesh::new's order
  unsigned int kind;            // 1 node out of range, 2 no positive volume, 3 flat
  unsigned int node;
  double value;
};

enum { BAD_RANGE = 1, BAD_VOLUME = 2, BAD_FLAT = 3 };

__device__ __forceinline__ unsigned tet_failure(const double* pos, size_t n, const uint32_t* t, unsigned* node,
                                                double* value) {
  for (int c = 0; c < 4; ++c)
    if (t[c] >= n) {
      *node = t[c];
      return BAD_RANGE;
    }
  const double* p[4] = {pos + 3 * (size_t)t[0], pos + 3 * (size_t)t[1], pos + 3 * (size_t)t[2], pos + 3 * (size_t)t[3]};
  const double vol = tet_volume(p[0], p[1], p[2], p[3]);
  if (isnan(vol) || vol <= 0.0) {
    *value = vol;
    return BAD_VOLUME;
  }
  const double rel = relative_volume(p[0], p[1], p[2], p[3], vol);
  if (isnan(rel) || rel < 1e-12) {
    *value = rel;
    return BAD_FLAT;
  }
  return 0;
}

__global__ void check_nodes_kernel(const double* __restrict__ pos, size_t n, Checks* out) {
  GRID_STRIDE(v, n) {
    if (!isfinite(pos[3 * v]) || !isfinite(pos[3 * v + 1]) || !isfinite(pos[3 * v + 2]))
      atomicMin(&out->nonfinite_node, (unsigned)v);
  }
}

__global__ void check_tets_kernel(const double* __restrict__ pos, size_t n, const uint32_t* __restrict__ tets,
                                  size_t ntets, uint32_t* __restrict__ used, Checks* out) {
  GRID_STRIDE(t, ntets) {
    unsigned node = 0;
    double value = 0.0;
    if (tet_failure(pos, n, tets + 4 * t, &node, &value)) {
      atomicMin(&out->bad_tet, (unsigned)t);
      continue;
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) used[tets[4 * t + c]] = 1u;
  }
}

__global__ void check_detail_kernel(const double* __restrict__ pos, size_t n, const uint32_t* __restrict__ tets,
                                    const uint32_t* __restrict__ used, size_t nused, Checks* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0 && out->bad_tet != 0xffffffffu) {
    unsigned node = 0;
    double value = 0.0;
    out->kind = tet_failure(pos, n, tets + 4 * (size_t)out->bad_tet, &node, &value);
    out->node = node;
    out->value = value;
  }
  if (out->bad_tet == 0xffffffffu) {
    GRID_STRIDE(v, nused) if (!used[v]) atomicMin(&out->unused_node, (unsigned)v);
  }
}

// ------------------------------------------------------------------ edges and midside nodes
__device__ __forceinline__ void edge_of(const uint32_t* t, int e, uint32_t* a, uint32_t* b) {
  const uint32_t x = t[kdEdge[e][0]], y = t[kdEdge[e][1]];
  *a = min(x, y);
  *b = max(x, y);
}

__global__ void edge_count_kernel(const uint32_t* __restrict__ tets, size_t ntets, uint32_t* __restrict__ count) {
  GRID_STRIDE(i, 6 * ntets) {
    uint32_t a, b;
    edge_of(tets + 4 * (i / 6), (int)(i % 6), &a, &b);
    atomicAdd(count + a, 1u);
  }
}

__global__ void edge_fill_kernel(const uint32_t* __restrict__ tets, size_t ntets, uint32_t* __restrict__ cursor,
                                 uint32_t* __restrict__ other) {
  GRID_STRIDE(i, 6 * ntets) {
    uint32_t a, b;
    edge_of(tets + 4 * (i / 6), (int)(i % 6), &a, &b);
    other[atomicAdd(cursor + a, 1u)] = b;
  }
}

// Sorts each node's bucket of larger edge ends and keeps each end once.
__global__ void edge_unique_kernel(const uint32_t* __restrict__ off, uint32_t* __restrict__ other,
                                   uint32_t* __restrict__ unique_count, size_t n) {
  GRID_STRIDE(a, n) {
    uint32_t* l = other + off[a];
    const uint32_t m = off[a + 1] - off[a];
    for (uint32_t i = 1; i < m; ++i) {
      const uint32_t x = l[i];
      uint32_t j = i;
      while (j > 0 && l[j - 1] > x) {
        l[j] = l[j - 1];
        --j;
      }
      l[j] = x;
    }
    uint32_t u = 0;
    for (uint32_t i = 0; i < m; ++i)
      if (u == 0 || l[i] != l[u - 1]) l[u++] = l[i];
    unique_count[a] = u;
  }
}

// The midside node of each unique edge (a, b): number n + its rank among the sorted edges, at
// 0.5 * (p + q) (quadratic.rs:40-52).
__global__ void midside_kernel(const uint32_t* __restrict__ off, const uint32_t* __restrict__ eoff,
                               const uint32_t* __restrict__ other, double* __restrict__ pos, size_t n) {
  GRID_STRIDE(a, n) {
    const uint32_t m = eoff[a + 1] - eoff[a];
    const double* p = pos + 3 * a;
    for (uint32_t j = 0; j < m; ++j) {
      const double* q = pos + 3 * (size_t)other[off[a] + j];
      double* out = pos + 3 * (n + eoff[a] + j);
      out[0] = 0.5 * (p[0] + q[0]);
      out[1] = 0.5 * (p[1] + q[1]);
      out[2] = 0.5 * (p[2] + q[2]);
    }
  }
}

__global__ void tet10_kernel(const uint32_t* __restrict__ corners, size_t ntets, const uint32_t* __restrict__ off,
                             const uint32_t* __restrict__ eoff, const uint32_t* __restrict__ other, uint32_t n,
                             uint32_t* __restrict__ tets10) {
  GRID_STRIDE(t, ntets) {
    const uint32_t* c = corners + 4 * t;
#pragma unroll
    for (int i = 0; i < 4; ++i) tets10[10 * t + i] = c[i];
    for (int e = 0; e < 6; ++e) {
      uint32_t a, b;
      edge_of(c, e, &a, &b);
      const uint32_t* l = other + off[a];
      uint32_t lo = 0, hi = eoff[a + 1] - eoff[a];
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (l[mid] < b)
          lo = mid + 1;
        else
          hi = mid;
      }
      tets10[10 * t + 4 + e] = n + eoff[a] + lo;
    }
  }
}

// ------------------------------------------------------------------ boundary faces
__device__ __forceinline__ void face_key(const uint32_t* t, int f, uint32_t (&k)[3]) {
  k[0] = t[kdFace[f][0]];
  k[1] = t[kdFace[f][1]];
  k[2] = t[kdFace[f][2]];
  uint32_t x;
  if (k[0] > k[1]) { x = k[0]; k[0] = k[1]; k[1] = x; }
  if (k[1] > k[2]) { x = k[1]; k[1] = k[2]; k[2] = x; }
  if (k[0] > k[1]) { x = k[0]; k[0] = k[1]; k[1] = x; }
}

__global__ void face_count_kernel(const uint32_t* __restrict__ tets, size_t ntets, uint32_t* __restrict__ count) {
  GRID_STRIDE(i, 4 * ntets) {
    uint32_t k[3];
    face_key(tets + 4 * (i / 4), (int)(i % 4), k);
    atomicAdd(count + k[0], 1u);
  }
}

__global__ void face_fill_kernel(const uint32_t* __restrict__ tets, size_t ntets, uint32_t* __restrict__ cursor,
                                 unsigned long long* __restrict__ rest, uint32_t* __restrict__ item) {
  GRID_STRIDE(i, 4 * ntets) {
    uint32_t k[3];
    face_key(tets + 4 * (i / 4), (int)(i % 4), k);
    const uint32_t at = atomicAdd(cursor + k[0], 1u);
    rest[at] = ((unsigned long long)k[1] << 32) | k[2];
    item[at] = (uint32_t)i;  // 4 tet + face
  }
}

// Sorts each bucket by (key, tet, face); counts the keys held by one face only and flags a key
// held by three or more.
__global__ void face_bucket_kernel(const uint32_t* __restrict__ off, unsigned long long* __restrict__ rest,
                                   uint32_t* __restrict__ item, uint32_t* __restrict__ single, Checks* checks, size_t n) {
  GRID_STRIDE(a, n) {
    unsigned long long* r = rest + off[a];
    uint32_t* it = item + off[a];
    const uint32_t m = off[a + 1] - off[a];
    for (uint32_t i = 1; i < m; ++i) {
      const unsigned long long x = r[i];
      const uint32_t y = it[i];
      uint32_t j = i;
      while (j > 0 && (r[j - 1] > x || (r[j - 1] == x && it[j - 1] > y))) {
        r[j] = r[j - 1];
        it[j] = it[j - 1];
        --j;
      }
      r[j] = x;
      it[j] = y;
    }
    uint32_t s = 0;
    for (uint32_t i = 0; i < m;) {
      uint32_t e = i + 1;
      while (e < m && r[e] == r[i]) ++e;
      if (e == i + 1) ++s;
      if (e >= i + 3) checks->non_manifold = 1u;
      i = e;
    }
    single[a] = s;
  }
}

__global__ void face_emit_kernel(const uint32_t* __restrict__ off, const unsigned long long* __restrict__ rest,
                                 const uint32_t* __restrict__ item, const uint32_t* __restrict__ soff,
                                 const uint32_t* __restrict__ tets10, sf_boundary_face* __restrict__ faces, size_t n) {
  GRID_STRIDE(a, n) {
    const unsigned long long* r = rest + off[a];
    const uint32_t* it = item + off[a];
    const uint32_t m = off[a + 1] - off[a];
    uint32_t o = soff[a];
    for (uint32_t i = 0; i < m;) {
      uint32_t e = i + 1;
      while (e < m && r[e] == r[i]) ++e;
      if (e == i + 1) {
        sf_boundary_face f;
        f.tet = it[i] / 4;
        f.face = it[i] % 4;
        for (int s = 0; s < 6; ++s) f.nodes[s] = tets10[10 * (size_t)f.tet + kdFace[f.face][s]];
        faces[o++] = f;
      }
      i = e;
    }
  }
}

// ------------------------------------------------------------------ host orchestration
// Device buffers of one build on its own non-blocking stream, from the device's stream-ordered
// pool; everything not handed to the mesh is freed on the stream when the build ends.
struct Build {
  int device = 0, prev = 0;
  cudaStream_t stream = nullptr;
  std::vector<void*> temps;
  cudaError_t err = cudaSuccess;
  ~Build() {
    for (void* p : temps) cudaFreeAsync(p, stream);
    if (stream) {
      cudaStreamSynchronize(stream);
      cudaStreamDestroy(stream);
    }
    cudaSetDevice(prev);
  }
  template <typename T>
  T* alloc(size_t count, bool keep = false) {
    void* p = nullptr;
    if (err == cudaSuccess) err = cudaMallocAsync(&p, std::max<size_t>(count, 1) * sizeof(T) + 64, stream);
    if (err != cudaSuccess) return nullptr;
    if (!keep) temps.push_back(p);
    return (T*)p;
  }
};

// Returns false (b.err set) when its scratch could not be allocated: the caller must not launch
// anything that reads `out`.
bool scan(Build& b, const uint32_t* in, uint32_t* out, size_t n) {
  const size_t nb = std::max<size_t>(1, (n + 1023) / 1024);
  uint32_t* sums = b.alloc<uint32_t>(nb);
  if (b.err) return false;
  if (n) scan_blocks_kernel<<<(unsigned)nb, 1024, 0, b.stream>>>(in, out, sums, n);
  else cudaMemsetAsync(sums, 0, sizeof(uint32_t), b.stream);
  scan_sums_kernel<<<1, 1024, 0, b.stream>>>(sums, n ? nb : 0, out + n);
  if (n) scan_add_kernel<<<grid_of(n), kT, 0, b.stream>>>(out, sums, n);
  return true;
}

struct DeviceMeshOwner : DeviceMesh {
  cudaStream_t stream = nullptr;
  ~DeviceMeshOwner() override {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    if (!stream) cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
    if (nodes) cudaFreeAsync(nodes, stream);
    if (tets) cudaFreeAsync(tets, stream);
    cudaStreamDestroy(stream);
    cudaSetDevice(prev);
  }
};

sf_status cuda_fail(cudaError_t e, const char* what);

// A scan whose scratch allocation failed: wait for the work already queued, report the failure.
sf_status scan_failed(Build& b) {
  cudaStreamSynchronize(b.stream);
  return cuda_fail(b.err, "scan");
}

sf_status cuda_fail(cudaError_t e, const char* what) {
  char msg[200];
  std::snprintf(msg, sizeof(msg), "%s: %s", what, cudaGetErrorString(e));
  cudaGetLastError();
  return fail(e == cudaErrorMemoryAllocation ? SF_DEVICE_MEMORY_BUDGET : SF_CUDA_ERROR, msg);
}

// TetMesh::new (checks) and QuadraticTetMesh::from_linear on `n` positions and `ntets` corner
// quadruples already on the device, into `out` (host arrays and the device mirror).
sf_status from_linear(Build& b, double* pos, size_t n, uint32_t* corners, size_t ntets, Mesh& out) {
  if (ntets == 0) return fail(SF_MESH_EMPTY, "the mesh has no tetrahedra");
  if (n >= 0xffffffffull || 6 * ntets >= 0xffffffffull)
    return fail(SF_INVALID_ARGUMENT, "the mesh is too large for 32-bit indices");
  cudaStream_t st = b.stream;
  Checks init;
  std::memset(&init, 0, sizeof(init));
  init.nonfinite_node = init.bad_tet = init.unused_node = 0xffffffffu;
  Checks* checks = b.alloc<Checks>(1);
  uint32_t* used = b.alloc<uint32_t>(n);
  if (b.err) return cuda_fail(b.err, "mesh build");
  cudaMemcpyAsync(checks, &init, sizeof(init), cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(used, 0, n * 4, st);
  check_nodes_kernel<<<grid_of(n), kT, 0, st>>>(pos, n, checks);
  check_tets_kernel<<<grid_of(ntets), kT, 0, st>>>(pos, n, corners, ntets, used, checks);
  check_detail_kernel<<<grid_of(n), kT, 0, st>>>(pos, n, corners, used, n, checks);
  Checks got;
  cudaMemcpyAsync(&got, checks, sizeof(got), cudaMemcpyDeviceToHost, st);
  if (cudaError_t e = cudaStreamSynchronize(st)) return cuda_fail(e, "mesh checks");
  // TetMesh::new's order: positions, then each tetrahedron in order, then unused nodes
  if (got.nonfinite_node != 0xffffffffu) {
    error_slot().node = got.nonfinite_node;
    return fail(SF_MESH_NON_FINITE_POSITION, "a node position is not finite");
  }
  if (got.bad_tet != 0xffffffffu) {
    error_slot().tet = got.bad_tet;
    if (got.kind == BAD_RANGE) {
      error_slot().node = got.node;
      return fail(SF_MESH_NODE_OUT_OF_RANGE, "a tetrahedron names a node that does not exist");
    }
    error_slot().value = got.value;
    if (got.kind == BAD_VOLUME) return fail(SF_MESH_DEGENERATE_TET, "a tetrahedron has no positive volume");
    return fail(SF_MESH_FLAT_TET, "a tetrahedron is flat to rounding");
  }
  if (got.unused_node != 0xffffffffu) {
    error_slot().node = got.unused_node;
    return fail(SF_MESH_UNUSED_NODE, "a node belongs to no tetrahedron");
  }
  // edges: bucket by the smaller end, sort and unique each bucket, number the midside nodes
  uint32_t* count = b.alloc<uint32_t>(n + 1);
  uint32_t* off = b.alloc<uint32_t>(n + 1);
  uint32_t* cursor = b.alloc<uint32_t>(n);
  uint32_t* other = b.alloc<uint32_t>(6 * ntets);
  uint32_t* ucount = b.alloc<uint32_t>(n + 1);
  uint32_t* eoff = b.alloc<uint32_t>(n + 1);
  if (b.err) return cuda_fail(b.err, "mesh build");
  cudaMemsetAsync(count, 0, n * 4, st);
  edge_count_kernel<<<grid_of(6 * ntets), kT, 0, st>>>(corners, ntets, count);
  if (!scan(b, count, off, n)) return scan_failed(b);
  cudaMemcpyAsync(cursor, off, n * 4, cudaMemcpyDeviceToDevice, st);
  edge_fill_kernel<<<grid_of(6 * ntets), kT, 0, st>>>(corners, ntets, cursor, other);
  edge_unique_kernel<<<grid_of(n), kT, 0, st>>>(off, other, ucount, n);
  if (!scan(b, ucount, eoff, n)) return scan_failed(b);
  uint32_t edges = 0;
  cudaMemcpyAsync(&edges, eoff + n, 4, cudaMemcpyDeviceToHost, st);
  if (cudaError_t e = cudaStreamSynchronize(st)) return cuda_fail(e, "mesh edges");
  if (b.err) return cuda_fail(b.err, "mesh build");
  const size_t nodes = n + edges;
  if (nodes >= 0xffffffffull) return fail(SF_INVALID_ARGUMENT, "the mesh is too large for 32-bit indices");
  // the ten-node arrays, kept on the device for the studies built from this mesh
  auto mirror = std::make_shared<DeviceMeshOwner>();
  mirror->device = b.device;
  mirror->nodes = b.alloc<double>(3 * nodes, true);
  mirror->tets = b.alloc<uint32_t>(10 * ntets, true);
  // On an early return the mirror frees its arrays on a stream of its own: the build's kernels
  // that write them must have finished first (declared after `mirror`, so it runs before).
  struct Drain {
    cudaStream_t st;
    bool armed = true;
    ~Drain() {
      if (armed) cudaStreamSynchronize(st);
    }
  } drain{st};
  if (b.err) return cuda_fail(b.err, "mesh build");
  cudaMemcpyAsync(mirror->nodes, pos, n * 24, cudaMemcpyDeviceToDevice, st);
  midside_kernel<<<grid_of(n), kT, 0, st>>>(off, eoff, other, mirror->nodes, n);
  tet10_kernel<<<grid_of(ntets), kT, 0, st>>>(corners, ntets, off, eoff, other, (uint32_t)n, mirror->tets);
  // boundary faces: bucket by the smallest corner, keys held by one tetrahedron in key order
  uint32_t* fcount = b.alloc<uint32_t>(n + 1);
  uint32_t* foff = b.alloc<uint32_t>(n + 1);
  unsigned long long* rest = b.alloc<unsigned long long>(4 * ntets);
  uint32_t* item = b.alloc<uint32_t>(4 * ntets);
  uint32_t* single = b.alloc<uint32_t>(n + 1);
  uint32_t* soff = b.alloc<uint32_t>(n + 1);
  if (b.err) return cuda_fail(b.err, "mesh build");
  cudaMemsetAsync(fcount, 0, n * 4, st);
  face_count_kernel<<<grid_of(4 * ntets), kT, 0, st>>>(corners, ntets, fcount);
  if (!scan(b, fcount, foff, n)) return scan_failed(b);
  cudaMemcpyAsync(cursor, foff, n * 4, cudaMemcpyDeviceToDevice, st);
  face_fill_kernel<<<grid_of(4 * ntets), kT, 0, st>>>(corners, ntets, cursor, rest, item);
  face_bucket_kernel<<<grid_of(n), kT, 0, st>>>(foff, rest, item, single, checks, n);
  if (!scan(b, single, soff, n)) return scan_failed(b);
  uint32_t nfaces = 0;
  unsigned int manifold = 0;
  cudaMemcpyAsync(&nfaces, soff + n, 4, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&manifold, &checks->non_manifold, 4, cudaMemcpyDeviceToHost, st);
  if (cudaError_t e = cudaStreamSynchronize(st)) return cuda_fail(e, "mesh faces");
  if (manifold) return fail(SF_MESH_NON_MANIFOLD_FACE, "a face is shared by more than two tetrahedra");
  sf_boundary_face* faces = b.alloc<sf_boundary_face>(nfaces);
  if (b.err) return cuda_fail(b.err, "mesh build");
  face_emit_kernel<<<grid_of(n), kT, 0, st>>>(foff, rest, item, soff, mirror->tets, faces, n);
  // host arrays
  out = Mesh();
  out.vertex_count = n;
  out.nodes.resize(nodes);
  out.tets.resize(ntets);
  out.corners.resize(ntets);
  out.faces.resize(nfaces);
  cudaMemcpyAsync(out.nodes.data(), mirror->nodes, nodes * 24, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(out.tets.data(), mirror->tets, ntets * 40, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(out.corners.data(), corners, ntets * 16, cudaMemcpyDeviceToHost, st);
  if (nfaces) cudaMemcpyAsync(out.faces.data(), faces, (size_t)nfaces * sizeof(sf_boundary_face), cudaMemcpyDeviceToHost, st);
  if (cudaError_t e = cudaStreamSynchronize(st)) return cuda_fail(e, "mesh copy");
  if (cudaError_t e = cudaGetLastError()) return cuda_fail(e, "mesh kernels");
  mirror->stream = nullptr;
  out.dev = mirror;
  drain.armed = false;  // the copies above synchronized the stream
  return SF_OK;
}

sf_status begin(Build& b, int device) {
  cudaGetDevice(&b.prev);
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count)
    return fail(SF_INVALID_ARGUMENT, "no such CUDA device");
  b.device = device;
  if (cudaError_t e = cudaSetDevice(device)) return cuda_fail(e, "set device");
  pool_setup(device);
  if (cudaError_t e = cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking)) return cuda_fail(e, "stream");
  return SF_OK;
}

sf_status check_box(const double size[3], const uint64_t div[3]) {
  for (int a = 0; a < 3; ++a)
    if (div[a] == 0) return fail(SF_MESH_INVALID_BOX, "each axis needs at least one division");
  for (int a = 0; a < 3; ++a)
    if (std::isnan(size[a]) || size[a] <= 0.0) return fail(SF_MESH_INVALID_BOX, "each box length must be positive");
  const double v = (double)(div[0] + 1) * (double)(div[1] + 1) * (double)(div[2] + 1);
  if (v > 4.0e9 || 6.0 * (double)div[0] * (double)div[1] * (double)div[2] > 7.0e8)
    return fail(SF_INVALID_ARGUMENT, "the box is too large for 32-bit indices");
  return SF_OK;
}

// ------------------------------------------------------------------ consistent traction load
// add_traction (crates/solidfem-elastic/src/loads.rs:10-41) on the device: the 6-point triangle
// rule's measure per face and point, then per node the sum over its traction faces in list order
// and over the points in order, starting from the node's nodal-force sum (build_load adds the
// forces first, study.rs:696-735): the host's accumulation order, so the same bits.
struct LoadFace {
  uint32_t nodes[6];
  double t[3];
};

__device__ __forceinline__ void triangle_point(int q, double* r, double* s, double* w) {
  const double TA = 0.091576213509771, TB = 0.445948490915965;
  const double WA = 0.109951743655322, WB = 0.223381589678011;
  const double pts[6][3] = {{TA, TA, WA}, {1.0 - 2.0 * TA, TA, WA}, {TA, 1.0 - 2.0 * TA, WA},
                            {TB, TB, WB}, {1.0 - 2.0 * TB, TB, WB}, {TB, 1.0 - 2.0 * TB, WB}};
  *r = pts[q][0];
  *s = pts[q][1];
  *w = pts[q][2];
}

__global__ void face_measure_kernel(const LoadFace* __restrict__ faces, size_t nfaces, const double* __restrict__ pos,
                                    double* __restrict__ measure) {
  GRID_STRIDE(i, 6 * nfaces) {
    const LoadFace& f = faces[i / 6];
    const int q = (int)(i % 6);
    double r, s, w;
    triangle_point(q, &r, &s, &w);
    const double l1 = 1.0 - r - s;
    const double dr[6] = {-(4.0 * l1 - 1.0), 4.0 * r - 1.0, 0.0, 4.0 * (l1 - r), 4.0 * s, -4.0 * s};
    const double ds[6] = {-(4.0 * l1 - 1.0), 0.0, 4.0 * s - 1.0, -4.0 * r, 4.0 * r, 4.0 * (l1 - s)};
    double tr[3] = {0, 0, 0}, ts[3] = {0, 0, 0};
    for (int n = 0; n < 6; ++n)
      for (int a = 0; a < 3; ++a) {
        const double p = pos[3 * (size_t)f.nodes[n] + a];
        tr[a] += dr[n] * p;
        ts[a] += ds[n] * p;
      }
    const double nm[3] = {tr[1] * ts[2] - tr[2] * ts[1], tr[2] * ts[0] - tr[0] * ts[2], tr[0] * ts[1] - tr[1] * ts[0]};
    const double length = sqrt(nm[0] * nm[0] + nm[1] * nm[1] + nm[2] * nm[2]);
    measure[i] = 0.5 * length * w;
  }
}

__global__ void load_count_kernel(const LoadFace* __restrict__ faces, size_t nfaces, uint32_t* __restrict__ count) {
  GRID_STRIDE(i, 6 * nfaces) atomicAdd(count + faces[i / 6].nodes[i % 6], 1u);
}

__global__ void load_fill_kernel(const LoadFace* __restrict__ faces, size_t nfaces, uint32_t* __restrict__ cursor,
                                 uint32_t* __restrict__ entry) {
  GRID_STRIDE(i, 6 * nfaces) entry[atomicAdd(cursor + faces[i / 6].nodes[i % 6], 1u)] = (uint32_t)i;  // 6 face + slot
}

// Node X: its force sum (or zero), then each traction face touching it in list order, each point
// in order: load += t[a] * v[slot] * measure (loads.rs:30-38).
__global__ void node_load_kernel(const LoadFace* __restrict__ faces, const double* __restrict__ measure,
                                 const uint32_t* __restrict__ off, uint32_t* __restrict__ entry,
                                 const uint32_t* __restrict__ forced, const double* __restrict__ force_sum,
                                 uint32_t nforced, double* __restrict__ load, size_t n) {
  GRID_STRIDE(x, n) {
    uint32_t* e = entry + off[x];
    const uint32_t m = off[x + 1] - off[x];
    for (uint32_t i = 1; i < m; ++i) {  // list order: ascending face
      const uint32_t v = e[i];
      uint32_t j = i;
      while (j > 0 && e[j - 1] > v) {
        e[j] = e[j - 1];
        --j;
      }
      e[j] = v;
    }
    double acc[3] = {0.0, 0.0, 0.0};
    uint32_t lo = 0, hi = nforced;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (forced[mid] < x)
        lo = mid + 1;
      else
        hi = mid;
    }
    if (lo < nforced && forced[lo] == x)
      for (int a = 0; a < 3; ++a) acc[a] = force_sum[3 * (size_t)lo + a];
    for (uint32_t i = 0; i < m; ++i) {
      const uint32_t face = e[i] / 6, slot = e[i] % 6;
      const double* t = faces[face].t;
      for (int q = 0; q < 6; ++q) {
        double r, s, w;
        triangle_point(q, &r, &s, &w);
        const double l1 = 1.0 - r - s;
        const double v[6] = {l1 * (2.0 * l1 - 1.0), r * (2.0 * r - 1.0), s * (2.0 * s - 1.0),
                             4.0 * l1 * r, 4.0 * r * s, 4.0 * s * l1};
        const double mq = measure[6 * (size_t)face + q];
        for (int a = 0; a < 3; ++a) acc[a] += t[a] * v[slot] * mq;
      }
    }
    for (int a = 0; a < 3; ++a) load[3 * x + a] = acc[a];
  }
}

// ------------------------------------------------------------------ the free-node pattern
// build_pattern on the device (assembly.rs:55-81, csr.rs:19-71): the node-to-element incidence
// (each node's elements ascending), each free row's node and assembly cursor, and each row's
// columns: the free numbers of the nodes of its node's elements, sorted and each kept once. A warp
// takes a row: its candidates (10 per element) go to shared memory, a bitonic sort orders them
// (fixed nodes, numbered 0xffffffff, sort last and are dropped), and a ballot keeps the first of
// each run. A row with more than kPatternCap candidates sends the whole mesh back to the host build.
constexpr int kPatternCap = 512;
constexpr int kPatternWarps = 8;

__global__ void incidence_count_kernel(const uint32_t* __restrict__ tets10, size_t n, uint32_t* __restrict__ count) {
  GRID_STRIDE(i, n) atomicAdd(count + tets10[i], 1u);
}

__global__ void incidence_fill_kernel(const uint32_t* __restrict__ tets10, size_t n, uint32_t* __restrict__ cursor,
                                      uint32_t* __restrict__ inc) {
  GRID_STRIDE(i, n) inc[atomicAdd(cursor + tets10[i], 1u)] = (uint32_t)(i / 10);
}

__global__ void incidence_sort_kernel(const uint32_t* __restrict__ start, uint32_t* __restrict__ inc, size_t nodes) {
  GRID_STRIDE(v, nodes) {
    uint32_t* l = inc + start[v];
    const uint32_t m = start[v + 1] - start[v];
    for (uint32_t i = 1; i < m; ++i) {
      const uint32_t x = l[i];
      uint32_t j = i;
      while (j > 0 && l[j - 1] > x) {
        l[j] = l[j - 1];
        --j;
      }
      l[j] = x;
    }
  }
}

__global__ void row_node_kernel(const uint32_t* __restrict__ free, const uint32_t* __restrict__ start, size_t nodes,
                                uint32_t* __restrict__ row_node, uint32_t* __restrict__ cursor) {
  GRID_STRIDE(v, nodes) {
    const uint32_t f = free[v];
    if (f != 0xffffffffu) {
      row_node[f] = (uint32_t)v;
      cursor[f] = start[v];  // the row's first element for the sliced assembly
    }
  }
}

template <bool FILL>
__global__ void __launch_bounds__(32 * kPatternWarps) pattern_rows_kernel(
    uint32_t rows, const uint32_t* __restrict__ row_node, const uint32_t* __restrict__ inc_start,
    const uint32_t* __restrict__ inc, const uint32_t* __restrict__ tets10, const uint32_t* __restrict__ free,
    const uint32_t* __restrict__ starts, uint32_t* __restrict__ out, unsigned* __restrict__ overflow) {
  __shared__ uint32_t buf[kPatternWarps][kPatternCap];
  const unsigned lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t* b = buf[w];
  for (uint32_t r = blockIdx.x * kPatternWarps + w; r < rows; r += gridDim.x * kPatternWarps) {
    const uint32_t node = row_node[r], k0 = inc_start[node], k1 = inc_start[node + 1];
    const uint32_t cand = 10 * (k1 - k0);
    if (cand > (uint32_t)kPatternCap) {
      if (lane == 0) {
        atomicOr(overflow, 1u);
        if (!FILL) out[r] = 0;
      }
      continue;
    }
    uint32_t p = 32;
    while (p < cand) p <<= 1;
    for (uint32_t i = lane; i < p; i += 32)
      b[i] = i < cand ? free[tets10[10 * (size_t)inc[k0 + i / 10] + i % 10]] : 0xffffffffu;
    __syncwarp();
    for (uint32_t k = 2; k <= p; k <<= 1)
      for (uint32_t j = k >> 1; j > 0; j >>= 1) {
        for (uint32_t i = lane; i < p; i += 32) {
          const uint32_t ixj = i ^ j;
          if (ixj > i) {
            const uint32_t x = b[i], y = b[ixj];
            if ((x > y) == ((i & k) == 0)) {
              b[i] = y;
              b[ixj] = x;
            }
          }
        }
        __syncwarp();
      }
    uint32_t count = 0;
    for (uint32_t i0 = 0; i0 < p; i0 += 32) {
      const uint32_t i = i0 + lane;
      const uint32_t v = b[i];
      const bool keep = v != 0xffffffffu && (i == 0 || b[i - 1] != v);
      const unsigned m = __ballot_sync(0xffffffffu, keep);
      if (FILL && keep) out[starts[r] + count + __popc(m & ((1u << lane) - 1u))] = v;
      count += __popc(m);
    }
    if (!FILL && lane == 0) out[r] = count;
    __syncwarp();
  }
}

}  // namespace

sf_status device_pattern(const Mesh& mesh, const vector<uint32_t>& free, size_t free_count, DevicePattern& out,
                         vector<uint32_t>& host_starts, bool* fallback) {
  *fallback = false;
  if (!mesh.dev) return fail(SF_INVALID_ARGUMENT, "the mesh has no device arrays");
  Build b;
  if (sf_status s = begin(b, mesh.dev->device)) return s;
  const size_t nn = mesh.nodes.size(), nt = 10 * mesh.tets.size();
  auto keep = [&](uint32_t** p, size_t count) {
    *p = b.alloc<uint32_t>(count, true);
    if (*p) out.allocations.push_back({*p, std::max<size_t>(count, 1) * 4 + 64});
  };
  auto release = [&]() {
    for (auto& a : out.allocations) cudaFreeAsync(a.first, b.stream);
    out = DevicePattern();
  };
  keep(&out.inc_start, nn + 1);
  keep(&out.inc, nt);
  keep(&out.row_node, free_count);
  keep(&out.cursor, free_count);
  keep(&out.starts, free_count + 1);
  uint32_t* dfree = b.alloc<uint32_t>(nn);
  uint32_t* count = b.alloc<uint32_t>(nn);
  uint32_t* cursor = b.alloc<uint32_t>(nn);
  uint32_t* rows = b.alloc<uint32_t>(free_count);
  unsigned* overflow = b.alloc<unsigned>(1);
  if (b.err) {
    release();
    return cuda_fail(b.err, "pattern");
  }
  cudaStream_t st = b.stream;
  cudaMemcpyAsync(dfree, free.data(), nn * 4, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(count, 0, nn * 4, st);
  cudaMemsetAsync(overflow, 0, 4, st);
  incidence_count_kernel<<<grid_of(nt), kT, 0, st>>>(mesh.dev->tets, nt, count);
  if (!scan(b, count, out.inc_start, nn)) {
    const sf_status e = scan_failed(b);
    release();
    return e;
  }
  cudaMemcpyAsync(cursor, out.inc_start, nn * 4, cudaMemcpyDeviceToDevice, st);
  incidence_fill_kernel<<<grid_of(nt), kT, 0, st>>>(mesh.dev->tets, nt, cursor, out.inc);
  incidence_sort_kernel<<<grid_of(nn), kT, 0, st>>>(out.inc_start, out.inc, nn);
  row_node_kernel<<<grid_of(nn), kT, 0, st>>>(dfree, out.inc_start, nn, out.row_node, out.cursor);
  const unsigned grid = (unsigned)std::max<size_t>(1, std::min<size_t>((free_count + kPatternWarps - 1) / kPatternWarps,
                                                                       148 * 16));
  pattern_rows_kernel<false><<<grid, 32 * kPatternWarps, 0, st>>>((uint32_t)free_count, out.row_node, out.inc_start,
                                                                  out.inc, mesh.dev->tets, dfree, nullptr, rows, overflow);
  if (!scan(b, rows, out.starts, free_count)) {
    const sf_status e = scan_failed(b);
    release();
    return e;
  }
  unsigned over = 0;
  uint32_t blocks = 0;
  cudaMemcpyAsync(&over, overflow, 4, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&blocks, out.starts + free_count, 4, cudaMemcpyDeviceToHost, st);
  if (cudaError_t e = cudaStreamSynchronize(st)) {
    release();
    return cuda_fail(e, "pattern");
  }
  if (over || b.err) {
    const cudaError_t err = b.err;
    release();
    if (err) return cuda_fail(err, "pattern");
    *fallback = true;
    return SF_OK;
  }
  out.blocks = blocks;
  keep(&out.cols, blocks);
  if (b.err) {
    const cudaError_t err = b.err;
    release();
    return cuda_fail(err, "pattern");
  }
  pattern_rows_kernel<true><<<grid, 32 * kPatternWarps, 0, st>>>((uint32_t)free_count, out.row_node, out.inc_start,
                                                                 out.inc, mesh.dev->tets, dfree, out.starts, out.cols,
                                                                 overflow);
  host_starts.resize(free_count + 1);
  cudaMemcpyAsync(host_starts.data(), out.starts, (free_count + 1) * 4, cudaMemcpyDeviceToHost, st);
  if (cudaError_t e = cudaStreamSynchronize(st)) {
    release();
    return cuda_fail(e, "pattern");
  }
  if (cudaError_t e = cudaGetLastError()) {
    release();
    return cuda_fail(e, "pattern");
  }
  return SF_OK;
}

sf_status device_traction_load(const Mesh& mesh, const vector<std::pair<sf_boundary_face, array<double, 3>>>& tractions,
                               vector<double>& load) {
  if (!mesh.dev) return fail(SF_INVALID_ARGUMENT, "the mesh has no device arrays");
  Build b;
  if (sf_status s = begin(b, mesh.dev->device)) return s;
  const size_t n = mesh.nodes.size(), nf = tractions.size();
  // the nodal forces already summed into `load` on the host, for the nodes that carry one
  vector<uint32_t> forced;
  vector<double> force_sum;
  for (size_t x = 0; x < n; ++x)
    if (load[3 * x] != 0.0 || load[3 * x + 1] != 0.0 || load[3 * x + 2] != 0.0 || std::signbit(load[3 * x]) ||
        std::signbit(load[3 * x + 1]) || std::signbit(load[3 * x + 2])) {
      forced.push_back((uint32_t)x);
      for (int a = 0; a < 3; ++a) force_sum.push_back(load[3 * x + a]);
    }
  vector<LoadFace> host(nf);
  for (size_t j = 0; j < nf; ++j) {
    for (int k = 0; k < 6; ++k) host[j].nodes[k] = tractions[j].first.nodes[k];
    for (int a = 0; a < 3; ++a) host[j].t[a] = tractions[j].second[a];
  }
  LoadFace* faces = b.alloc<LoadFace>(nf);
  double* measure = b.alloc<double>(6 * nf);
  uint32_t* count = b.alloc<uint32_t>(n + 1);
  uint32_t* off = b.alloc<uint32_t>(n + 1);
  uint32_t* cursor = b.alloc<uint32_t>(n);
  uint32_t* entry = b.alloc<uint32_t>(6 * nf);
  uint32_t* dforced = b.alloc<uint32_t>(forced.size());
  double* dsum = b.alloc<double>(force_sum.size());
  double* dload = b.alloc<double>(3 * n);
  if (b.err) return cuda_fail(b.err, "traction load");
  cudaStream_t st = b.stream;
  if (nf) cudaMemcpyAsync(faces, host.data(), nf * sizeof(LoadFace), cudaMemcpyHostToDevice, st);
  if (!forced.empty()) {
    cudaMemcpyAsync(dforced, forced.data(), forced.size() * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dsum, force_sum.data(), force_sum.size() * 8, cudaMemcpyHostToDevice, st);
  }
  cudaMemsetAsync(count, 0, n * 4, st);
  face_measure_kernel<<<grid_of(6 * nf), kT, 0, st>>>(faces, nf, mesh.dev->nodes, measure);
  load_count_kernel<<<grid_of(6 * nf), kT, 0, st>>>(faces, nf, count);
  if (!scan(b, count, off, n)) return scan_failed(b);
  cudaMemcpyAsync(cursor, off, n * 4, cudaMemcpyDeviceToDevice, st);
  load_fill_kernel<<<grid_of(6 * nf), kT, 0, st>>>(faces, nf, cursor, entry);
  node_load_kernel<<<grid_of(n), kT, 0, st>>>(faces, measure, off, entry, dforced, dsum, (uint32_t)forced.size(), dload,
                                              n);
  cudaMemcpyAsync(load.data(), dload, 3 * n * 8, cudaMemcpyDeviceToHost, st);
  if (cudaError_t e = cudaStreamSynchronize(st)) return cuda_fail(e, "traction load");
  if (cudaError_t e = cudaGetLastError()) return cuda_fail(e, "traction load");
  return SF_OK;
}

sf_status build_box_mesh_device(const double origin[3], const double size[3], const uint64_t div[3], int device,
                                Mesh& out) {
  if (sf_status s = check_box(size, div)) return s;
  Build b;
  if (sf_status s = begin(b, device)) return s;
  Box box;
  for (int a = 0; a < 3; ++a) {
    box.o[a] = origin[a];
    box.s[a] = size[a];
    box.d[a] = div[a];
  }
  const size_t n = (div[0] + 1) * (div[1] + 1) * (div[2] + 1), ntets = 6 * div[0] * div[1] * div[2];
  double* pos = b.alloc<double>(3 * n);
  uint32_t* tets = b.alloc<uint32_t>(4 * ntets);
  if (b.err) return cuda_fail(b.err, "mesh build");
  box_vertices_kernel<<<grid_of(n), kT, 0, b.stream>>>(box, pos, n);
  box_tets_kernel<<<grid_of(ntets), kT, 0, b.stream>>>(box, tets, ntets);
  return from_linear(b, pos, n, tets, ntets, out);
}

sf_status build_part_mesh_device(const double* const lines[3], const uint64_t counts[3], uint64_t wall_cells,
                                 int device, Mesh& out) {
  uint64_t cells[3];
  for (int a = 0; a < 3; ++a) {
    if (!lines[a] || counts[a] < 2) return fail(SF_MESH_INVALID_BOX, "each axis needs at least one cell");
    cells[a] = counts[a] - 1;
  }
  const double unit_size[3] = {(double)cells[0], (double)cells[1], (double)cells[2]};
  if (sf_status s = check_box(unit_size, cells)) return s;
  Build b;
  if (sf_status s = begin(b, device)) return s;
  // the unit grid: box_tet_mesh([0; 3], cells, cells), part.rs:146-150
  Box unit;
  for (int a = 0; a < 3; ++a) {
    unit.o[a] = 0.0;
    unit.s[a] = unit_size[a];
    unit.d[a] = cells[a];
  }
  const size_t nv = (cells[0] + 1) * (cells[1] + 1) * (cells[2] + 1), nt = 6 * cells[0] * cells[1] * cells[2];
  double* upos = b.alloc<double>(3 * nv);
  uint32_t* keep = b.alloc<uint32_t>(nt + 1);
  uint32_t* at = b.alloc<uint32_t>(nt + 1);
  unsigned int* first = b.alloc<unsigned int>(nv);
  double* dl[3];
  for (int a = 0; a < 3; ++a) dl[a] = b.alloc<double>(counts[a]);
  if (b.err) return cuda_fail(b.err, "mesh build");
  for (int a = 0; a < 3; ++a) cudaMemcpyAsync(dl[a], lines[a], counts[a] * 8, cudaMemcpyHostToDevice, b.stream);
  box_vertices_kernel<<<grid_of(nv), kT, 0, b.stream>>>(unit, upos, nv);
  PartCells g{cells[1], cells[2], wall_cells};
  part_keep_kernel<<<grid_of(nt), kT, 0, b.stream>>>(unit, g, upos, keep, nt);
  if (!scan(b, keep, at, nt)) return scan_failed(b);
  uint32_t kept_count = 0;
  cudaMemcpyAsync(&kept_count, at + nt, 4, cudaMemcpyDeviceToHost, b.stream);
  if (cudaError_t e = cudaStreamSynchronize(b.stream)) return cuda_fail(e, "part cells");
  if (b.err) return cuda_fail(b.err, "mesh build");
  if (kept_count == 0) return fail(SF_MESH_EMPTY, "the mesh has no tetrahedra");
  uint32_t* kept = b.alloc<uint32_t>(4 * (size_t)kept_count);
  uint32_t* mark = b.alloc<uint32_t>(4 * (size_t)kept_count + 1);
  uint32_t* rank = b.alloc<uint32_t>(4 * (size_t)kept_count + 1);
  if (b.err) return cuda_fail(b.err, "mesh build");
  cudaMemsetAsync(first, 0xff, nv * 4, b.stream);
  cudaMemsetAsync(mark, 0, 4 * (size_t)kept_count * 4, b.stream);
  part_compact_kernel<<<grid_of(nt), kT, 0, b.stream>>>(unit, keep, at, kept, first, nt);
  part_mark_kernel<<<grid_of(nv), kT, 0, b.stream>>>(first, mark, nv);
  if (!scan(b, mark, rank, 4 * (size_t)kept_count)) return scan_failed(b);
  uint32_t used = 0;
  cudaMemcpyAsync(&used, rank + 4 * (size_t)kept_count, 4, cudaMemcpyDeviceToHost, b.stream);
  if (cudaError_t e = cudaStreamSynchronize(b.stream)) return cuda_fail(e, "part vertices");
  double* pos = b.alloc<double>(3 * (size_t)used);
  if (b.err) return cuda_fail(b.err, "mesh build");
  part_positions_kernel<<<grid_of(nv), kT, 0, b.stream>>>(unit, first, rank, dl[0], dl[1], dl[2], pos, nv);
  part_remap_kernel<<<grid_of(4 * (size_t)kept_count), kT, 0, b.stream>>>(first, rank, kept, 4 * (size_t)kept_count);
  return from_linear(b, pos, used, kept, kept_count, out);
}

sf_status build_linear_mesh_device(const double* positions, uint64_t n, const uint32_t* tets, uint64_t ntets,
                                   int device, Mesh& out) {
  Build b;
  if (sf_status s = begin(b, device)) return s;
  if (ntets == 0) return fail(SF_MESH_EMPTY, "the mesh has no tetrahedra");
  double* pos = b.alloc<double>(3 * std::max<uint64_t>(n, 1));
  uint32_t* t = b.alloc<uint32_t>(4 * ntets);
  if (b.err) return cuda_fail(b.err, "mesh build");
  if (n) cudaMemcpyAsync(pos, positions, n * 24, cudaMemcpyHostToDevice, b.stream);
  cudaMemcpyAsync(t, tets, ntets * 16, cudaMemcpyHostToDevice, b.stream);
  return from_linear(b, pos, n, t, ntets, out);
}

}  // namespace sf
