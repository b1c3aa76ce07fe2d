// The FP64 numeric phases of the multigrid setup on the device: block-diagonal inversion, block
// norms for the join pass, the power iteration for lambda_max(D^-1 A), prolongator smoothing,
// A P and the Galerkin product P^T (A P) (crates/solidfem-solve/src/multigrid/setup.rs:269-321,
// 390-449, 527-647; transfer.rs:108-238; block.rs:186-245, 379-404).
//
// Built with -fmad=false and IEEE division and square root. Every output value is one thread's
// sequential sum over its contributions in the order the reference's serial loops visit them, so
// the device hierarchy equals the reference's to the bit. Parallelism comes from independent
// outputs: a thread owns one block row of the power iteration, one block of P, of A P or of the
// coarse matrix. The order-dependent graph work (strength, aggregation, tentative prolongator)
// and every sparsity pattern are built on the host (setup.cpp); only values live here.
//
// The one sequential reduction, the power iteration's norm (block.rs:398-404 sums the squares in
// index order), runs on the host (setup.cpp), where a single core adds a dependent chain of
// doubles several times faster than one GPU thread; the products stay here.
#include <cuda_runtime.h>

#include <atomic>

#include <algorithm>

#include "device.h"

namespace sf {

namespace {

constexpr double kRankTolerance = 1e-10;  // transfer.rs:12
constexpr size_t kTentativeMaxSmem = 200 * 1024;  // an aggregate's rows x 6 modes, staged whole

const int kT = 256;

int grid_for(size_t n) { return (int)std::max<size_t>(1, std::min<size_t>((n + kT - 1) / kT, 148 * 32)); }

// C += A B for row-major dense blocks, the loop order of block.rs:229-245.
template <int AR, int MID, int BC>
__device__ __forceinline__ void add_product(double* out, const double* a, const double* b) {
#pragma unroll
  for (int r = 0; r < AR; ++r)
#pragma unroll
    for (int m = 0; m < MID; ++m) {
      double s = a[r * MID + m];
#pragma unroll
      for (int c = 0; c < BC; ++c) out[r * BC + c] += s * b[m * BC + c];
    }
}

__device__ __forceinline__ bool contains(const uint32_t* b, const uint32_t* e, uint32_t v) {
  while (b < e) {
    const uint32_t* mid = b + (e - b) / 2;
    if (*mid < v)
      b = mid + 1;
    else if (*mid > v)
      e = mid;
    else
      return true;
  }
  return false;
}

// Cholesky-based inverse of an SPD block (block.rs:186-224).
template <int N>
__device__ bool invert_spd(const double* in, double* out, double* pivot) {
  double lower[N * N];
  double inv[N * N];
#pragma unroll
  for (int i = 0; i < N * N; ++i) lower[i] = inv[i] = 0.0;
  for (int i = 0; i < N; ++i)
    for (int j = 0; j <= i; ++j) {
      double sum = in[i * N + j];
      for (int k = 0; k < j; ++k) sum -= lower[i * N + k] * lower[j * N + k];
      if (i == j) {
        if (!isfinite(sum) || sum <= 0.0) {
          *pivot = sum;
          return false;
        }
        lower[i * N + j] = sqrt(sum);
      } else {
        lower[i * N + j] = sum / lower[j * N + j];
      }
    }
  for (int c = 0; c < N; ++c)
    for (int i = c; i < N; ++i) {
      double sum = i == c ? 1.0 : 0.0;
      for (int k = c; k < i; ++k) sum -= lower[i * N + k] * inv[k * N + c];
      inv[i * N + c] = sum / lower[i * N + i];
    }
  for (int i = 0; i < N; ++i)
    for (int j = 0; j < N; ++j) {
      double sum = 0.0;
      for (int k = i > j ? i : j; k < N; ++k) sum += inv[k * N + i] * inv[k * N + j];
      out[i * N + j] = sum;
    }
  return true;
}

template <int N>
__global__ void inverse_diagonal_kernel(uint32_t rows, const uint32_t* __restrict__ starts,
                                        const uint32_t* __restrict__ cols, const double* __restrict__ vals,
                                        double* __restrict__ inv, unsigned long long* bad, double* __restrict__ pivots) {
  for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < rows; row += gridDim.x * blockDim.x) {
    const uint32_t* b = cols + starts[row];
    const uint32_t* e = cols + starts[row + 1];
    const uint32_t* lo = b;
    const uint32_t* hi = e;
    while (lo < hi) {
      const uint32_t* mid = lo + (hi - lo) / 2;
      if (*mid < row)
        lo = mid + 1;
      else
        hi = mid;
    }
    double pivot = 0.0;
    bool ok = lo != e && *lo == row &&
              invert_spd<N>(vals + (size_t)(lo - cols) * N * N, inv + (size_t)row * N * N, &pivot);
    if (!ok) {
      pivots[row] = pivot;
      atomicMin(bad, (unsigned long long)row);
    }
  }
}

template <int LEN>
__global__ void block_norms_kernel(size_t blocks, const double* __restrict__ vals, double* __restrict__ out) {
  for (size_t b = blockIdx.x * (size_t)blockDim.x + threadIdx.x; b < blocks; b += (size_t)gridDim.x * blockDim.x) {
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < LEN; ++i) {
      double v = vals[b * LEN + i];
      s += v * v;
    }
    out[b] = sqrt(s);
  }
}

// v = src / d, element by element.
__global__ void scale_kernel(size_t n, const double* __restrict__ src, double d, double* __restrict__ v) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    v[i] = src[i] / d;
}

// s2 = D^-1 (A v) for one block row per thread, in the order of setup.rs:404-432.
// One power step s2 = D^-1 (A v) (setup.rs:390-449). Lane p of a team of N lanes owns component
// p of a block row: its sum runs over the row's blocks in column order and, inside a block, over
// q in order, one running sum, as the reference's serial loop; the team's N sums then meet by
// shuffles for D^-1 y, again summed in q order. A warp holds 32 / N teams (10 rows of 3, 5 of
// 6), so a block's N value rows are read by N neighbouring lanes.
template <int N>
__global__ void power_step_kernel(uint32_t rows, const uint32_t* __restrict__ starts, const uint32_t* __restrict__ cols,
                                  const double* __restrict__ vals, const double* __restrict__ inv,
                                  const double* __restrict__ v, double* __restrict__ s2) {
  constexpr uint32_t kTeams = 32 / N;
  const uint32_t lane = threadIdx.x & 31, team = lane / N, p = lane - team * N;
  const bool on = team < kTeams;
  const uint32_t warps = blockDim.x >> 5;
  const uint32_t warp0 = blockIdx.x * warps + (threadIdx.x >> 5);
  for (uint32_t base = warp0 * kTeams; base < rows; base += gridDim.x * warps * kTeams) {
    const uint32_t row = base + team;
    const bool live = on && row < rows;
    double y = 0.0;
    if (live) {
      for (uint32_t at = starts[row]; at < starts[row + 1]; ++at) {
        const double* b = vals + (size_t)at * N * N + (size_t)p * N;
        const double* x = v + (size_t)cols[at] * N;
        double sum = y;
#pragma unroll
        for (int q = 0; q < N; ++q) sum += b[q] * x[q];
        y = sum;
      }
    }
    const uint32_t first = team * N;
    double yq[N];
#pragma unroll
    for (int q = 0; q < N; ++q) yq[q] = __shfl_sync(0xffffffffu, y, (first + q) & 31);
    if (live) {
      const double* d = inv + (size_t)row * N * N + (size_t)p * N;
      double sum = 0.0;
#pragma unroll
      for (int q = 0; q < N; ++q) sum += d[q] * yq[q];
      s2[(size_t)row * N + p] = sum;
    }
  }
}

// Row r of a union pattern: the sorted distinct columns inner_cols[k] over the inner rows j of r's
// outer list (j = r itself first when `self`); with inner_starts null each j has the one column
// inner_cols[j]. A warp per row sets the columns' bits in its own bitmap of `words` words in shared
// memory, then walks the bitmap in order: 32 words at a time, a warp prefix sum of their popcounts
// places each word's set bits. The count pass (out_starts null) writes the row's column count to
// out[r]; the fill pass writes the columns at out[out_starts[r] ..]. Every bit is cleared after use.
__global__ void union_rows_kernel(uint32_t rows, uint32_t words, const uint32_t* __restrict__ outer_starts,
                                  const uint32_t* __restrict__ outer_idx, int self,
                                  const uint32_t* __restrict__ inner_starts, const uint32_t* __restrict__ inner_cols,
                                  const uint32_t* __restrict__ out_starts, uint32_t* __restrict__ out) {
  extern __shared__ uint32_t union_bits[];
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  uint32_t* bm = union_bits + (size_t)warp * words;
  for (uint32_t i = lane; i < words; i += 32) bm[i] = 0;
  __syncwarp();
  for (uint32_t r = blockIdx.x * warps + warp; r < rows; r += gridDim.x * warps) {
    const uint32_t o0 = outer_starts[r], n = outer_starts[r + 1] - o0 + (self ? 1u : 0u);
    for (uint32_t t = lane; t < n; t += 32) {
      const uint32_t j = self ? (t == 0 ? r : outer_idx[o0 + t - 1]) : outer_idx[o0 + t];
      if (inner_starts) {
        for (uint32_t k = inner_starts[j]; k < inner_starts[j + 1]; ++k) {
          const uint32_t c = inner_cols[k];
          atomicOr(&bm[c >> 5], 1u << (c & 31));
        }
      } else {
        const uint32_t c = inner_cols[j];
        atomicOr(&bm[c >> 5], 1u << (c & 31));
      }
    }
    __syncwarp();
    const uint32_t base = out_starts ? out_starts[r] : 0u;
    uint32_t total = 0;
    for (uint32_t w0 = 0; w0 < words; w0 += 32) {
      const uint32_t w = w0 + lane;
      uint32_t bits = w < words ? bm[w] : 0u;
      const uint32_t cnt = (uint32_t)__popc(bits);
      uint32_t inc = cnt;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(full, inc, o);
        if (lane >= o) inc += v;
      }
      if (out_starts) {
        uint32_t at = base + total + (inc - cnt);
        while (bits) {
          out[at++] = w * 32u + (uint32_t)(__ffs(bits) - 1);
          bits &= bits - 1;
        }
      }
      if (w < words) bm[w] = 0u;
      total += __shfl_sync(full, inc, 31);
    }
    if (!out_starts && lane == 0) out[r] = total;
    __syncwarp();
  }
}

// The block row of each entry of a block pattern.
__global__ void entry_rows_kernel(uint32_t rows, const uint32_t* __restrict__ starts, uint32_t* __restrict__ out) {
  for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < rows; row += gridDim.x * blockDim.x)
    for (uint32_t j = starts[row]; j < starts[row + 1]; ++j) out[j] = row;
}

// One block of P = T - omega D^-1 A_f T (transfer.rs:108-152): A's blocks whose column is the row
// or a smoothing neighbour act on that column's tentative block; the others are lumped onto the
// row's own (src = row). Contributions to this block's coarse column add in A's column order.
template <int N>
__global__ void smooth_kernel(size_t entries, const uint32_t* __restrict__ entry_row, const uint32_t* __restrict__ p_cols,
                              const uint32_t* __restrict__ a_starts, const uint32_t* __restrict__ a_cols,
                              const double* __restrict__ a_vals, const uint32_t* __restrict__ n_starts,
                              const uint32_t* __restrict__ n_cols, const uint32_t* __restrict__ aggregate,
                              const double* __restrict__ t_vals, const double* __restrict__ inv, double omega,
                              double* __restrict__ p_vals) {
  constexpr int L = N * 6;
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < entries; j += (size_t)gridDim.x * blockDim.x) {
    const uint32_t row = entry_row[j], c = p_cols[j];
    const uint32_t* nb = n_cols + n_starts[row];
    const uint32_t* ne = n_cols + n_starts[row + 1];
    double acc[L];
#pragma unroll
    for (int i = 0; i < L; ++i) acc[i] = 0.0;
    for (uint32_t at = a_starts[row]; at < a_starts[row + 1]; ++at) {
      const uint32_t col = a_cols[at];
      const uint32_t src = (col == row || contains(nb, ne, col)) ? col : row;
      if (aggregate[src] != c) continue;
      add_product<N, N, 6>(acc, a_vals + (size_t)at * N * N, t_vals + (size_t)src * L);
    }
    const double* d = inv + (size_t)row * N * N;
    const double* t = t_vals + (size_t)row * L;
    const bool own = c == aggregate[row];
    double* out = p_vals + j * L;
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        double s = 0.0;
#pragma unroll
        for (int m = 0; m < N; ++m) s += d[r * N + m] * acc[m * 6 + q];
        double tv = own ? t[r * 6 + q] : 0.0;
        out[r * 6 + q] = tv - omega * s;
      }
  }
}

// One block of A P (transfer.rs:155-169): A's blocks in column order, each times the blocks of
// P's row at that column whose coarse column is this block's.
template <int N>
__global__ void product_kernel(size_t entries, const uint32_t* __restrict__ entry_row, const uint32_t* __restrict__ ap_cols,
                               const uint32_t* __restrict__ a_starts, const uint32_t* __restrict__ a_cols,
                               const double* __restrict__ a_vals, const uint32_t* __restrict__ p_starts,
                               const uint32_t* __restrict__ p_cols, const double* __restrict__ p_vals,
                               double* __restrict__ ap_vals) {
  constexpr int L = N * 6;
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < entries; j += (size_t)gridDim.x * blockDim.x) {
    const uint32_t row = entry_row[j], c = ap_cols[j];
    double acc[L];
#pragma unroll
    for (int i = 0; i < L; ++i) acc[i] = 0.0;
    for (uint32_t at = a_starts[row]; at < a_starts[row + 1]; ++at) {
      const uint32_t col = a_cols[at];
      for (uint32_t in = p_starts[col]; in < p_starts[col + 1]; ++in) {
        const uint32_t pc = p_cols[in];
        if (pc < c) continue;
        if (pc == c) add_product<N, N, 6>(acc, a_vals + (size_t)at * N * N, p_vals + (size_t)in * L);
        break;
      }
    }
    double* out = ap_vals + j * L;
#pragma unroll
    for (int i = 0; i < L; ++i) out[i] = acc[i];
  }
}

// One block of P^T (A P) (transfer.rs:173-238): the fine rows of P's column in ascending order,
// each P block transposed times the A P block of that fine row at this block's column; a zero on
// the diagonal of a diagonal block becomes one (finish_level, setup.rs:650-695).
template <int N>
__global__ void galerkin_kernel(size_t entries, const uint32_t* __restrict__ entry_row, const uint32_t* __restrict__ c_cols,
                                const uint32_t* __restrict__ pt_starts, const uint32_t* __restrict__ pt_rows,
                                const uint32_t* __restrict__ pt_at, const double* __restrict__ p_vals,
                                const uint32_t* __restrict__ ap_starts, const uint32_t* __restrict__ ap_cols,
                                const double* __restrict__ ap_vals, double* __restrict__ c_vals) {
  constexpr int L = N * 6;
  for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < entries; j += (size_t)gridDim.x * blockDim.x) {
    const uint32_t crow = entry_row[j], c = c_cols[j];
    double acc[36];
#pragma unroll
    for (int i = 0; i < 36; ++i) acc[i] = 0.0;
    for (uint32_t k = pt_starts[crow]; k < pt_starts[crow + 1]; ++k) {
      const uint32_t fine_row = pt_rows[k];
      const uint32_t* b = ap_cols + ap_starts[fine_row];
      const uint32_t* e = ap_cols + ap_starts[fine_row + 1];
      const uint32_t* lo = b;
      const uint32_t* hi = e;
      while (lo < hi) {
        const uint32_t* mid = lo + (hi - lo) / 2;
        if (*mid < c)
          lo = mid + 1;
        else
          hi = mid;
      }
      if (lo == e || *lo != c) continue;
      const double* pb = p_vals + (size_t)pt_at[k] * L;
      const double* ab = ap_vals + (size_t)(lo - ap_cols) * L;
#pragma unroll
      for (int r = 0; r < 6; ++r)
#pragma unroll
        for (int m = 0; m < N; ++m) {
          double s = pb[m * 6 + r];
#pragma unroll
          for (int q = 0; q < 6; ++q) acc[r * 6 + q] += s * ab[m * 6 + q];
        }
    }
    if (crow == c)
#pragma unroll
      for (int d = 0; d < 6; ++d)
        if (acc[d * 6 + d] == 0.0) acc[d * 6 + d] = 1.0;
    double* out = c_vals + j * 36;
#pragma unroll
    for (int i = 0; i < 36; ++i) out[i] = acc[i];
  }
}

// The tentative prolongator (setup.rs:327-386, orthonormalize_aggregate, transfer.rs:19-68): per
// aggregate, its members' rows of the near-null modes, orthonormalised column by column with two
// Gram-Schmidt passes against the earlier columns; a column whose remainder falls to
// RANK_TOLERANCE of its original norm is zeroed. One warp per aggregate stages the aggregate's
// rows (members in order, rb rows each, 6 modes) in shared memory; lane 0 runs every sum of the
// reference's loops in their order (sequential over the aggregate's rows), and the lanes share the
// element-wise updates, each of which depends only on its own entry. So T (written back at the
// members' own rows) and the coarse near-null space (the projections and remainders, 6 x 6 per
// aggregate) carry the host loops' bits.
__global__ void __launch_bounds__(32) tentative_kernel(uint32_t aggregates, int rb,
                                                       const uint32_t* __restrict__ member_starts,
                                                       const uint32_t* __restrict__ members,
                                                       const double* __restrict__ near_null, double* __restrict__ t,
                                                       double* __restrict__ coarse) {
  extern __shared__ double local[];  // lrows x 6
  const uint32_t a = blockIdx.x;
  const unsigned lane = threadIdx.x;
  if (a >= aggregates) return;
  const uint32_t m0 = member_starts[a];
  const uint32_t lrows = (member_starts[a + 1] - m0) * (uint32_t)rb;
  auto slot = [&](uint32_t r) { return ((size_t)members[m0 + r / rb] * rb + r % rb) * 6; };
  for (uint32_t r = lane; r < lrows; r += 32) {
    const size_t at = slot(r);
    for (int k = 0; k < 6; ++k) local[r * 6 + k] = near_null[at + k];
  }
  __syncwarp();
  double* c = coarse + (size_t)a * 36;
  if (lane == 0)
    for (int i = 0; i < 36; ++i) c[i] = 0.0;
  auto column_norm = [&](int col) {  // lane 0's sequential sum, broadcast
    double s = 0.0;
    if (lane == 0)
      for (uint32_t r = 0; r < lrows; ++r) s += local[r * 6 + col] * local[r * 6 + col];
    return __shfl_sync(0xffffffffu, sqrt(s), 0);
  };
  for (int col = 0; col < 6; ++col) {
    const double original = column_norm(col);
    for (int pass = 0; pass < 2; ++pass)
      for (int prev = 0; prev < col; ++prev) {
        double proj = 0.0;
        if (lane == 0) {
          for (uint32_t r = 0; r < lrows; ++r) proj += local[r * 6 + prev] * local[r * 6 + col];
          c[prev * 6 + col] += proj;
        }
        proj = __shfl_sync(0xffffffffu, proj, 0);
        for (uint32_t r = lane; r < lrows; r += 32) local[r * 6 + col] -= proj * local[r * 6 + prev];
        __syncwarp();
      }
    const double rem = column_norm(col);
    const bool drop = original == 0.0 || rem <= kRankTolerance * original;
    for (uint32_t r = lane; r < lrows; r += 32) local[r * 6 + col] = drop ? 0.0 : local[r * 6 + col] / rem;
    if (lane == 0) c[col * 6 + col] = drop ? 0.0 : rem;
    __syncwarp();
  }
  for (uint32_t r = lane; r < lrows; r += 32) {
    const size_t at = slot(r);
    for (int k = 0; k < 6; ++k) t[at + k] = local[r * 6 + k];
  }
}

// The free nodes' rigid-body modes (free_rigid_body_modes, rigid_modes.rs:36-83) about the centre
// and scale the host summed: for free block row r (node row_node[r]) the three rows
// [1 0 0 0 z -y], [0 1 0 -z 0 x], [0 0 1 y -x 0] of the scaled offsets, (row, mode) at 6 row + mode.
__global__ void rigid_modes_kernel(uint32_t rows, const uint32_t* __restrict__ row_node, const double* __restrict__ nodes,
                                   double cx, double cy, double cz, double scale, double* __restrict__ modes) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  const double* p = nodes + (size_t)row_node[r] * 3;
  const double x = (p[0] - cx) * scale, y = (p[1] - cy) * scale, z = (p[2] - cz) * scale;
  const double v[18] = {1, 0, 0, 0, z, -y, 0, 1, 0, -z, 0, x, 0, 0, 1, y, -x, 0};
  double* m = modes + (size_t)r * 18;
  for (int i = 0; i < 18; ++i) m[i] = v[i];
}

// ------------------------------------------------------------ the coarsest level's dense factor
// DenseCholesky (block.rs:307-374) and the explicit inverse L^-T L^-1 the cycle applies. The
// factor is computed right-looking in panels of kPanel columns: a panel kernel finishes its
// columns (the diagonal, then every entry below it, each summing its last terms in ascending k),
// a trailing kernel subtracts the panel's terms from the rest of the lower triangle, again in
// ascending k. Every entry therefore subtracts L[i][k] L[j][k] for k = 0, 1, ... in order from its
// original value, exactly the reference's left-looking loop, so the factor has the host loops'
// bits. Row-major n x n in device memory (the lower triangle holds the factor).
constexpr int kPanel = 32;

__global__ void dense_from_blocks_kernel(uint32_t rows, int rb, int cb, const uint32_t* __restrict__ starts,
                                         const uint32_t* __restrict__ cols, const double* __restrict__ vals, size_t n,
                                         double* __restrict__ f) {
  const uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= rows) return;
  for (uint32_t at = starts[row]; at < starts[row + 1]; ++at) {
    const size_t col = cols[at];
    for (int p = 0; p < rb; ++p)
      for (int q = 0; q < cb; ++q) f[((size_t)row * rb + p) * n + col * cb + q] = vals[(size_t)at * rb * cb + p * cb + q];
  }
}

// Columns [j0, j0 + kPanel) of the factor, one block; the first non-positive pivot is recorded
// (its column and value) and the factor stops there.
__global__ void __launch_bounds__(1024) cholesky_panel_kernel(size_t n, size_t j0, double* __restrict__ f,
                                                              unsigned long long* bad, double* pivot) {
  __shared__ double d;
  __shared__ int failed;
  if (threadIdx.x == 0) failed = *bad != ~0ull;
  __syncthreads();
  if (failed) return;
  const size_t j1 = j0 + kPanel < n ? j0 + kPanel : n;
  for (size_t j = j0; j < j1; ++j) {
    if (threadIdx.x == 0) {
      double sum = f[j * n + j];
      for (size_t k = j0; k < j; ++k) sum -= f[j * n + k] * f[j * n + k];
      if (!isfinite(sum) || sum <= 0.0) {
        *bad = j;
        *pivot = sum;
        failed = 1;
      } else {
        d = sqrt(sum);
        f[j * n + j] = d;
      }
    }
    __syncthreads();
    if (failed) return;
    for (size_t i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
      double s = f[i * n + j];
      for (size_t k = j0; k < j; ++k) s -= f[i * n + k] * f[j * n + k];
      f[i * n + j] = s / d;
    }
    __syncthreads();
  }
}

// The panel's terms off every entry (i, j) of the lower triangle right of it, k ascending.
__global__ void cholesky_trailing_kernel(size_t n, size_t j0, double* __restrict__ f, const unsigned long long* bad) {
  if (*bad != ~0ull) return;
  const size_t j1 = j0 + kPanel;
  const size_t m = n - j1;  // trailing size
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= m * m) return;
  const size_t i = j1 + e / m, j = j1 + e % m;
  if (j > i) return;
  double s = f[i * n + j];
  for (size_t k = j0; k < j1; ++k) s -= f[i * n + k] * f[j * n + k];
  f[i * n + j] = s;
}

// Column c of L^-1 by forward substitution on the unit vector (the host loop's order).
__global__ void lower_inverse_kernel(size_t n, const double* __restrict__ f, double* __restrict__ li) {
  const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  for (size_t i = c; i < n; ++i) {
    double s = i == c ? 1.0 : 0.0;
    for (size_t k = c; k < i; ++k) s -= f[i * n + k] * li[k * n + c];
    li[i * n + c] = s / f[i * n + i];
  }
}

// A^-1 = L^-T L^-1, entry (i, j) summing k from max(i, j) up.
__global__ void gram_inverse_kernel(size_t n, const double* __restrict__ li, double* __restrict__ out) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n * n) return;
  const size_t i = e / n, j = e % n;
  double s = 0.0;
  for (size_t k = i > j ? i : j; k < n; ++k) s += li[k * n + i] * li[k * n + j];
  out[e] = s;
}

template <typename S>
__global__ void convert_kernel(size_t n, const double* __restrict__ in, S* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (S)in[i];
}

// R = P^T block by block: R block o is P block src[o] transposed (rb x cb into cb x rb).
template <typename S>
__global__ void transpose_blocks_kernel(size_t blocks, int rb, int cb, const uint32_t* __restrict__ src,
                                        const double* __restrict__ in, S* __restrict__ out) {
  const int len = rb * cb;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < blocks; o += (size_t)gridDim.x * blockDim.x) {
    const double* p = in + (size_t)src[o] * len;
    S* t = out + o * len;
    for (int a = 0; a < rb; ++a)
      for (int b = 0; b < cb; ++b) t[b * rb + a] = (S)p[a * cb + b];
  }
}

// Fills a SELL-32 copy from a block CSR matrix (f64 values, converted to S): one thread per slice
// lane places its row's columns and values at their chunked positions; padding stays zero.
template <typename S, int LEN>
__global__ void sell_fill_kernel(size_t slots, const uint32_t* __restrict__ sell_rows, const uint32_t* __restrict__ sell_len,
                                 const uint32_t* __restrict__ sell_start, uint32_t nrows,
                                 const uint32_t* __restrict__ starts, const uint32_t* __restrict__ cols,
                                 const double* __restrict__ in, uint32_t* __restrict__ out_cols, S* __restrict__ out) {
  constexpr int U = sell_chunk_blocks(LEN, (int)sizeof(S));
  constexpr int VEC = 16 / (int)sizeof(S);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < slots; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t row = sell_rows[i];
    if (row >= nrows) continue;
    const uint32_t s = (uint32_t)(i / 32), t = (uint32_t)(i % 32), n = sell_len[i], b0 = starts[row];
    for (uint32_t k = 0; k < n; ++k) {
      const size_t q = sell_start[s] + 32 * (k - k % U) + t * U + k % U;
      out_cols[q] = cols[b0 + k];
#pragma unroll
      for (int e = 0; e < LEN; ++e) out[sell_value_offset(q, LEN, U, VEC, e)] = (S)in[(size_t)(b0 + k) * LEN + e];
    }
  }
}

// Fills a split-row copy of a 6 x CB block CSR matrix: lane t = 6 m + p of a slice places row p
// of each block of its block row as a 1 x CB block at its chunked SELL position; the lane with
// p = 0 also places the block's column in the block row's shared column chunk.
template <typename S, int CB>
__global__ void split_fill_kernel(size_t slots, const uint32_t* __restrict__ sell_rows, const uint32_t* __restrict__ sell_len,
                                  const uint32_t* __restrict__ sell_start, uint32_t nrows,
                                  const uint32_t* __restrict__ starts, const uint32_t* __restrict__ cols,
                                  const double* __restrict__ in, uint32_t* __restrict__ out_cols, S* __restrict__ out) {
  constexpr int U = sell_chunk_blocks(CB, (int)sizeof(S));
  constexpr int VEC = 16 / (int)sizeof(S);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < slots; i += (size_t)gridDim.x * blockDim.x) {
    const uint32_t row = sell_rows[i];
    if (row >= nrows) continue;
    const uint32_t s = (uint32_t)(i / 32), t = (uint32_t)(i % 32), m = t / 6, p = t % 6;
    const uint32_t n = sell_len[i], b0 = starts[row];
    const size_t cbase = (size_t)(sell_start[s] / 32) * kSplitRowsPerSlice + (size_t)m * U;
    for (uint32_t k = 0; k < n; ++k) {
      const uint32_t c = k / U, u = k % U;
      const size_t q = sell_start[s] + 32 * (size_t)(c * U) + t * U + u;
      if (p == 0) out_cols[cbase + (size_t)kSplitRowsPerSlice * U * c + u] = cols[b0 + k];
#pragma unroll
      for (int e = 0; e < CB; ++e)
        out[sell_value_offset(q, CB, U, VEC, e)] = (S)in[(size_t)(b0 + k) * 6 * CB + p * CB + e];
    }
  }
}

// Copies listed blocks out of (gather) or back into (scatter) a block array.
__global__ void gather_blocks_kernel(size_t count, int len, const uint32_t* __restrict__ idx,
                                     const double* __restrict__ in, double* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count * len; i += (size_t)gridDim.x * blockDim.x)
    out[i] = in[(size_t)idx[i / len] * len + i % len];
}
__global__ void scatter_blocks_kernel(size_t count, int len, const uint32_t* __restrict__ idx,
                                      const double* __restrict__ in, double* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count * len; i += (size_t)gridDim.x * blockDim.x)
    out[(size_t)idx[i / len] * len + i % len] = in[i];
}
__global__ void set_values_kernel(size_t count, const uint32_t* __restrict__ idx, const double* __restrict__ vals,
                                  double* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
    out[idx[i]] = vals[i];
}

}  // namespace

sf_status setup_gather_blocks(cudaStream_t st, size_t count, int len, const uint32_t* idx, const double* in,
                              double* out) {
  if (count == 0) return SF_OK;
  gather_blocks_kernel<<<grid_for(count * len), kT, 0, st>>>(count, len, idx, in, out);
  return cuda_check(cudaGetLastError(), "gather blocks");
}

sf_status setup_scatter_blocks(cudaStream_t st, size_t count, int len, const uint32_t* idx, const double* in,
                               double* out) {
  if (count == 0) return SF_OK;
  scatter_blocks_kernel<<<grid_for(count * len), kT, 0, st>>>(count, len, idx, in, out);
  return cuda_check(cudaGetLastError(), "scatter blocks");
}

sf_status setup_set_values(cudaStream_t st, size_t count, const uint32_t* idx, const double* vals, double* out) {
  if (count == 0) return SF_OK;
  set_values_kernel<<<grid_for(count), kT, 0, st>>>(count, idx, vals, out);
  return cuda_check(cudaGetLastError(), "set values");
}

sf_status setup_inverse_diagonal(cudaStream_t st, uint32_t rows, int rb, const uint32_t* starts, const uint32_t* cols,
                                 const double* vals, double* inv, unsigned long long* bad, double* pivots) {
  if (rows == 0) return SF_OK;
  if (rb == 3)
    inverse_diagonal_kernel<3><<<grid_for(rows), kT, 0, st>>>(rows, starts, cols, vals, inv, bad, pivots);
  else
    inverse_diagonal_kernel<6><<<grid_for(rows), kT, 0, st>>>(rows, starts, cols, vals, inv, bad, pivots);
  return cuda_check(cudaGetLastError(), "inverse diagonal");
}

sf_status setup_block_norms(cudaStream_t st, size_t blocks, int len, const double* vals, double* out) {
  if (blocks == 0) return SF_OK;
  if (len == 9)
    block_norms_kernel<9><<<grid_for(blocks), kT, 0, st>>>(blocks, vals, out);
  else
    block_norms_kernel<36><<<grid_for(blocks), kT, 0, st>>>(blocks, vals, out);
  return cuda_check(cudaGetLastError(), "block norms");
}

sf_status setup_power_step(cudaStream_t st, uint32_t rows, int rb, const uint32_t* starts, const uint32_t* cols,
                           const double* vals, const double* inv, const double* v, double* s2) {
  if (rows == 0) return SF_OK;
  if (rb == 3)
    power_step_kernel<3><<<grid_for((size_t)rows * 32 / 10), kT, 0, st>>>(rows, starts, cols, vals, inv, v, s2);
  else
    power_step_kernel<6><<<grid_for((size_t)rows * 32 / 5), kT, 0, st>>>(rows, starts, cols, vals, inv, v, s2);
  return cuda_check(cudaGetLastError(), "power step");
}

sf_status setup_scale(cudaStream_t st, size_t n, const double* src, double d, double* v) {
  if (n == 0) return SF_OK;
  scale_kernel<<<grid_for(n), kT, 0, st>>>(n, src, d, v);
  return cuda_check(cudaGetLastError(), "scale");
}

sf_status setup_union_rows(cudaStream_t st, uint32_t rows, uint32_t width, const uint32_t* outer_starts,
                           const uint32_t* outer_idx, bool self, const uint32_t* inner_starts,
                           const uint32_t* inner_cols, const uint32_t* out_starts, uint32_t* out) {
  const uint32_t words = (width + 31) / 32;
  const size_t per_warp = (size_t)std::max<uint32_t>(words, 1) * 4;
  const size_t limit = 200 * 1024;
  if (per_warp > limit) return fail(SF_INVALID_ARGUMENT, "union pattern wider than one warp's bitmap");
  const int warps = (int)std::max<size_t>(1, std::min<size_t>(8, limit / per_warp));
  const size_t smem = per_warp * warps;
  if (rows == 0) return SF_OK;
  const void* k = (const void*)union_rows_kernel;
  if (smem > 48 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)limit);
  const int grid = (int)std::max<size_t>(1, std::min<size_t>((rows + warps - 1) / warps, 148 * 16));
  union_rows_kernel<<<grid, 32 * warps, smem, st>>>(rows, words, outer_starts, outer_idx, self ? 1 : 0, inner_starts,
                                                    inner_cols, out_starts, out);
  return cuda_check(cudaGetLastError(), "union pattern");
}

// Strong neighbours by geometry (aggregate.rs:53-69): a thread per row takes the squared distance
// to each other column term for term (no contraction, as on the host), the row's closest one, and
// keeps the columns within reach^2 times it. out_starts null: each row's count into out and its
// closest distance into closest; else the strong columns in column order at out[out_starts[row]].
__global__ void strength_kernel(uint32_t rows, const uint32_t* __restrict__ starts, const uint32_t* __restrict__ cols,
                                const double* __restrict__ pos, double limit_scale, double* __restrict__ closest,
                                const uint32_t* __restrict__ out_starts, uint32_t* __restrict__ out) {
  for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < rows; row += gridDim.x * blockDim.x) {
    const double* p = pos + 3 * (size_t)row;
    const uint32_t a0 = starts[row], a1 = starts[row + 1];
    double c = 1.7976931348623157e308;
    for (uint32_t at = a0; at < a1; ++at) {
      const uint32_t col = cols[at];
      if (col == row) continue;
      const double* q = pos + 3 * (size_t)col;
      const double dx = q[0] - p[0], dy = q[1] - p[1], dz = q[2] - p[2];
      const double d = dx * dx + dy * dy + dz * dz;
      c = d < c ? d : c;  // std::min(c, d)
    }
    const double limit = limit_scale * c;
    uint32_t n = 0;
    for (uint32_t at = a0; at < a1; ++at) {
      const uint32_t col = cols[at];
      if (col == row) continue;
      const double* q = pos + 3 * (size_t)col;
      const double dx = q[0] - p[0], dy = q[1] - p[1], dz = q[2] - p[2];
      if (dx * dx + dy * dy + dz * dz <= limit) {
        if (out_starts) out[out_starts[row] + n] = col;
        ++n;
      }
    }
    if (!out_starts) {
      closest[row] = c;
      out[row] = n;
    }
  }
}

sf_status setup_strength(cudaStream_t st, uint32_t rows, const uint32_t* starts, const uint32_t* cols, const double* pos,
                         double limit_scale, double* closest, const uint32_t* out_starts, uint32_t* out) {
  if (rows == 0) return SF_OK;
  strength_kernel<<<grid_for(rows), kT, 0, st>>>(rows, starts, cols, pos, limit_scale, closest, out_starts, out);
  return cuda_check(cudaGetLastError(), "strength");
}

sf_status setup_entry_rows(cudaStream_t st, uint32_t rows, const uint32_t* starts, uint32_t* out) {
  if (rows == 0) return SF_OK;
  entry_rows_kernel<<<grid_for(rows), kT, 0, st>>>(rows, starts, out);
  return cuda_check(cudaGetLastError(), "entry rows");
}

sf_status setup_rigid_modes(cudaStream_t st, uint32_t rows, const uint32_t* row_node, const double* nodes,
                            const double center[3], double scale, double* modes) {
  if (rows == 0) return SF_OK;
  rigid_modes_kernel<<<(rows + 255) / 256, 256, 0, st>>>(rows, row_node, nodes, center[0], center[1], center[2], scale,
                                                         modes);
  return cuda_check(cudaGetLastError(), "rigid modes");
}

sf_status setup_dense_inverse(cudaStream_t st, uint32_t rows, int rb, const uint32_t* starts, const uint32_t* cols,
                              const double* vals, size_t n, double* work, double* li, double* inverse,
                              unsigned long long* bad, double* pivot) {
  if (n == 0) return SF_OK;
  cudaMemsetAsync(work, 0, n * n * 8, st);
  cudaMemsetAsync(li, 0, n * n * 8, st);
  dense_from_blocks_kernel<<<(rows + 127) / 128, 128, 0, st>>>(rows, rb, rb, starts, cols, vals, n, work);
  for (size_t j0 = 0; j0 < n; j0 += kPanel) {
    cholesky_panel_kernel<<<1, 1024, 0, st>>>(n, j0, work, bad, pivot);
    if (j0 + kPanel < n) {
      const size_t m = n - j0 - kPanel;
      cholesky_trailing_kernel<<<(unsigned)((m * m + 255) / 256), 256, 0, st>>>(n, j0, work, bad);
    }
  }
  lower_inverse_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(n, work, li);
  gram_inverse_kernel<<<(unsigned)((n * n + 255) / 256), 256, 0, st>>>(n, li, inverse);
  return cuda_check(cudaGetLastError(), "dense inverse");
}

sf_status setup_tentative(cudaStream_t st, size_t aggregates, int rb, size_t max_members, const uint32_t* member_starts,
                          const uint32_t* members, const double* near_null, double* t, double* coarse) {
  if (aggregates == 0) return SF_OK;
  const size_t smem = max_members * (size_t)rb * 6 * sizeof(double);
  if (smem > kTentativeMaxSmem) return fail(SF_INVALID_ARGUMENT, "an aggregate too large for the tentative kernel");
  static std::atomic<uint64_t> opted{0};  // the opt-in above 48 KB, once per device
  int dev = 0;
  cudaGetDevice(&dev);
  const uint64_t bit = dev < 64 ? 1ull << dev : 0;
  if (smem > 48 * 1024 && (!bit || !(opted.load() & bit))) {
    cudaFuncSetAttribute(tentative_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTentativeMaxSmem);
    opted.fetch_or(bit);
  }
  tentative_kernel<<<(unsigned)aggregates, 32, smem, st>>>((uint32_t)aggregates, rb, member_starts, members, near_null,
                                                           t, coarse);
  return cuda_check(cudaGetLastError(), "tentative");
}

sf_status setup_smooth(cudaStream_t st, int rb, size_t entries, const uint32_t* entry_row, const uint32_t* p_cols,
                       const uint32_t* a_starts, const uint32_t* a_cols, const double* a_vals, const uint32_t* n_starts,
                       const uint32_t* n_cols, const uint32_t* aggregate, const double* t_vals, const double* inv,
                       double omega, double* p_vals) {
  if (entries == 0) return SF_OK;
  if (rb == 3)
    smooth_kernel<3><<<grid_for(entries), kT, 0, st>>>(entries, entry_row, p_cols, a_starts, a_cols, a_vals, n_starts,
                                                       n_cols, aggregate, t_vals, inv, omega, p_vals);
  else
    smooth_kernel<6><<<grid_for(entries), kT, 0, st>>>(entries, entry_row, p_cols, a_starts, a_cols, a_vals, n_starts,
                                                       n_cols, aggregate, t_vals, inv, omega, p_vals);
  return cuda_check(cudaGetLastError(), "smooth");
}

sf_status setup_product(cudaStream_t st, int rb, size_t entries, const uint32_t* entry_row, const uint32_t* ap_cols,
                        const uint32_t* a_starts, const uint32_t* a_cols, const double* a_vals, const uint32_t* p_starts,
                        const uint32_t* p_cols, const double* p_vals, double* ap_vals) {
  if (entries == 0) return SF_OK;
  if (rb == 3)
    product_kernel<3><<<grid_for(entries), kT, 0, st>>>(entries, entry_row, ap_cols, a_starts, a_cols, a_vals,
                                                        p_starts, p_cols, p_vals, ap_vals);
  else
    product_kernel<6><<<grid_for(entries), kT, 0, st>>>(entries, entry_row, ap_cols, a_starts, a_cols, a_vals,
                                                        p_starts, p_cols, p_vals, ap_vals);
  return cuda_check(cudaGetLastError(), "product");
}

sf_status setup_galerkin(cudaStream_t st, int rb, size_t entries, const uint32_t* entry_row, const uint32_t* c_cols,
                         const uint32_t* pt_starts, const uint32_t* pt_rows, const uint32_t* pt_at, const double* p_vals,
                         const uint32_t* ap_starts, const uint32_t* ap_cols, const double* ap_vals, double* c_vals) {
  if (entries == 0) return SF_OK;
  if (rb == 3)
    galerkin_kernel<3><<<grid_for(entries), kT, 0, st>>>(entries, entry_row, c_cols, pt_starts, pt_rows, pt_at, p_vals,
                                                         ap_starts, ap_cols, ap_vals, c_vals);
  else
    galerkin_kernel<6><<<grid_for(entries), kT, 0, st>>>(entries, entry_row, c_cols, pt_starts, pt_rows, pt_at, p_vals,
                                                         ap_starts, ap_cols, ap_vals, c_vals);
  return cuda_check(cudaGetLastError(), "galerkin");
}

template <typename S>
sf_status setup_convert(cudaStream_t st, size_t n, const double* in, S* out) {
  if (n == 0) return SF_OK;
  convert_kernel<S><<<grid_for(n), kT, 0, st>>>(n, in, out);
  return cuda_check(cudaGetLastError(), "convert");
}
template sf_status setup_convert<float>(cudaStream_t, size_t, const double*, float*);
template sf_status setup_convert<double>(cudaStream_t, size_t, const double*, double*);

template <typename S>
sf_status setup_transpose_blocks(cudaStream_t st, size_t blocks, int rb, int cb, const uint32_t* src, const double* in,
                                 S* out) {
  if (blocks == 0) return SF_OK;
  transpose_blocks_kernel<S><<<grid_for(blocks), kT, 0, st>>>(blocks, rb, cb, src, in, out);
  return cuda_check(cudaGetLastError(), "transpose blocks");
}
template sf_status setup_transpose_blocks<float>(cudaStream_t, size_t, int, int, const uint32_t*, const double*, float*);
template sf_status setup_transpose_blocks<double>(cudaStream_t, size_t, int, int, const uint32_t*, const double*, double*);

template <typename S>
sf_status setup_sell_fill(cudaStream_t st, size_t slots, int len, const uint32_t* sell_rows, const uint32_t* sell_len,
                          const uint32_t* sell_start, uint32_t nrows, const uint32_t* starts, const uint32_t* cols,
                          const double* in, uint32_t* out_cols, S* out) {
  if (slots == 0) return SF_OK;
  switch (len) {
    case 9:
      sell_fill_kernel<S, 9><<<grid_for(slots), kT, 0, st>>>(slots, sell_rows, sell_len, sell_start, nrows, starts, cols,
                                                            in, out_cols, out);
      break;
    case 18:
      sell_fill_kernel<S, 18><<<grid_for(slots), kT, 0, st>>>(slots, sell_rows, sell_len, sell_start, nrows, starts, cols,
                                                             in, out_cols, out);
      break;
    case 36:
      sell_fill_kernel<S, 36><<<grid_for(slots), kT, 0, st>>>(slots, sell_rows, sell_len, sell_start, nrows, starts, cols,
                                                             in, out_cols, out);
      break;
    default: return fail(SF_INVALID_ARGUMENT, "unsupported block size for the SELL layout");
  }
  return cuda_check(cudaGetLastError(), "SELL fill");
}
template <typename S>
sf_status setup_split_fill(cudaStream_t st, size_t slots, int cb, const uint32_t* sell_rows, const uint32_t* sell_len,
                           const uint32_t* sell_start, uint32_t nrows, const uint32_t* starts, const uint32_t* cols,
                           const double* in, uint32_t* out_cols, S* out) {
  if (slots == 0) return SF_OK;
  if (cb == 3)
    split_fill_kernel<S, 3><<<grid_for(slots), kT, 0, st>>>(slots, sell_rows, sell_len, sell_start, nrows, starts, cols,
                                                           in, out_cols, out);
  else if (cb == 6)
    split_fill_kernel<S, 6><<<grid_for(slots), kT, 0, st>>>(slots, sell_rows, sell_len, sell_start, nrows, starts, cols,
                                                           in, out_cols, out);
  else
    return fail(SF_INVALID_ARGUMENT, "unsupported block size for the split-row layout");
  return cuda_check(cudaGetLastError(), "split fill");
}
template sf_status setup_split_fill<float>(cudaStream_t, size_t, int, const uint32_t*, const uint32_t*, const uint32_t*,
                                           uint32_t, const uint32_t*, const uint32_t*, const double*, uint32_t*, float*);
template sf_status setup_split_fill<double>(cudaStream_t, size_t, int, const uint32_t*, const uint32_t*, const uint32_t*,
                                            uint32_t, const uint32_t*, const uint32_t*, const double*, uint32_t*, double*);

template sf_status setup_sell_fill<float>(cudaStream_t, size_t, int, const uint32_t*, const uint32_t*, const uint32_t*,
                                          uint32_t, const uint32_t*, const uint32_t*, const double*, uint32_t*, float*);
template sf_status setup_sell_fill<double>(cudaStream_t, size_t, int, const uint32_t*, const uint32_t*, const uint32_t*,
                                           uint32_t, const uint32_t*, const uint32_t*, const double*, uint32_t*, double*);

}  // namespace sf
