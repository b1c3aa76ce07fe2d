// The solve path on sm_100a: the block-CSR products of the V-cycle and the conjugate gradient,
// the fused Chebyshev smoother, restriction through the stored transpose, prolongation, the
// coarsest level's dense solve and the FP64 conjugate gradient with fixed-order reductions.
//
// Layout: a block row's values are one contiguous slab of row-major blocks. A warp owns a block
// row; it stages the slab into shared memory with 16-byte coalesced streaming loads and then each
// lane multiplies one block, so the value stream is read once, fully coalesced, and x (held in
// L2) is gathered per block. Sums are reduced across the warp with a fixed butterfly, so every run
// gives the same bits. Each kernel reads the solver's status word first and returns at once when
// the solve has ended, so a batch of iterations can be enqueued (or replayed as a CUDA graph)
// without a host round trip per iteration.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>

#include "device.h"

namespace sf {

namespace {

const unsigned kFull = 0xffffffffu;
const int kThreads = 256;
const int kWarps = kThreads / 32;
const int kBlocksPerPass = 32;

template <typename S, int RB, int CB>
struct Slab {
  static constexpr int kLen = RB * CB;
  static constexpr int kBytes = kBlocksPerPass * kLen * (int)sizeof(S) + 32;
  static constexpr int kInt4 = (kBytes + 15) / 16;
};

__device__ __forceinline__ int stage_slab(const void* src, int bytes, int4* dst, int lane) {
  uintptr_t a = reinterpret_cast<uintptr_t>(src);
  uintptr_t a0 = a & ~uintptr_t(15);
  int off = (int)(a - a0);
  int chunks = (off + bytes + 15) >> 4;
  const int4* g = reinterpret_cast<const int4*>(a0);
  for (int c = lane; c < chunks; c += 32) dst[c] = __ldcs(g + c);
  return off;
}

template <typename V>
__device__ __forceinline__ V ld_vec(const V* p) {
  return __ldg(p);
}

// The RB sums of one block row of A x, in every lane of the warp.
template <typename S, typename V, int RB, int CB>
__device__ __forceinline__ void warp_row_product(const uint32_t* __restrict__ starts,
                                                 const uint32_t* __restrict__ cols,
                                                 const S* __restrict__ vals,
                                                 const V* __restrict__ x, uint32_t row, int lane,
                                                 int4* sbuf, V acc[RB]) {
  constexpr int LEN = RB * CB;
#pragma unroll
  for (int p = 0; p < RB; ++p) acc[p] = V(0);
  uint32_t s = starts[row], e = starts[row + 1];
  for (uint32_t base = s; base < e; base += kBlocksPerPass) {
    int count = (int)min((uint32_t)kBlocksPerPass, e - base);
    int off = stage_slab(vals + (size_t)base * LEN, count * LEN * (int)sizeof(S), sbuf, lane);
    uint32_t c = lane < count ? __ldcs(cols + base + lane) : 0u;
    __syncwarp();
    if (lane < count) {
      const S* blk = reinterpret_cast<const S*>(reinterpret_cast<const char*>(sbuf) + off) + lane * LEN;
      V xv[CB];
#pragma unroll
      for (int q = 0; q < CB; ++q) xv[q] = ld_vec(x + (size_t)c * CB + q);
#pragma unroll
      for (int p = 0; p < RB; ++p)
#pragma unroll
        for (int q = 0; q < CB; ++q) acc[p] += V(blk[p * CB + q]) * xv[q];
    }
    __syncwarp();
  }
#pragma unroll
  for (int p = 0; p < RB; ++p)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[p] += __shfl_xor_sync(kFull, acc[p], o);
}

template <typename V, int RB>
__device__ __forceinline__ V select_lane(const V acc[RB], int lane) {
  V v = acc[0];
#pragma unroll
  for (int p = 1; p < RB; ++p)
    if (lane == p) v = acc[p];
  return v;
}

enum { OP_SET = 0, OP_RESIDUAL = 1, OP_ADD = 2 };

// y = A x (OP_SET), y = b - A x (OP_RESIDUAL), y = y + A x (OP_ADD).
template <typename S, typename V, int RB, int CB, int OP>
__global__ void __launch_bounds__(kThreads) bsr_kernel(uint32_t rows, const uint32_t* __restrict__ starts,
                                                       const uint32_t* __restrict__ cols,
                                                       const S* __restrict__ vals, const V* __restrict__ x,
                                                       V* __restrict__ y, const V* __restrict__ b,
                                                       const int* __restrict__ status) {
  if (*status != ST_ACTIVE) return;
  extern __shared__ int4 smem[];
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int4* sbuf = smem + warp * Slab<S, RB, CB>::kInt4;
  uint32_t nw = gridDim.x * kWarps;
  for (uint32_t row = blockIdx.x * kWarps + warp; row < rows; row += nw) {
    V acc[RB];
    warp_row_product<S, V, RB, CB>(starts, cols, vals, x, row, lane, sbuf, acc);
    if (lane < RB) {
      V sum = select_lane<V, RB>(acc, lane);
      size_t i = (size_t)row * RB + lane;
      if (OP == OP_SET) y[i] = sum;
      if (OP == OP_RESIDUAL) y[i] = b[i] - sum;
      if (OP == OP_ADD) y[i] = y[i] + sum;
    }
  }
}

// One Chebyshev step fused with its product (cycle.rs:611-650): ad = A d_old; r -= ad;
// z = D^-1 r; d_new = keep d_old + step z; x += d_new. With `outer` set (the last step of the
// post-smoother) the smoothed correction is added straight into the level's x:
// outer += (x + d_new), the reference's post_x += d then x += post_x (cycle.rs:533-536).
template <typename S, typename V, int RB>
__global__ void __launch_bounds__(kThreads) cheb_step_kernel(
    uint32_t rows, const uint32_t* __restrict__ starts, const uint32_t* __restrict__ cols,
    const S* __restrict__ vals, const S* __restrict__ dinv, const V* __restrict__ d_old,
    V* __restrict__ d_new, V* __restrict__ r, V* __restrict__ x, V* __restrict__ outer, V keep, V step,
    const int* __restrict__ status) {
  if (*status != ST_ACTIVE) return;
  extern __shared__ int4 smem[];
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int4* sbuf = smem + warp * Slab<S, RB, RB>::kInt4;
  uint32_t nw = gridDim.x * kWarps;
  for (uint32_t row = blockIdx.x * kWarps + warp; row < rows; row += nw) {
    V acc[RB];
    warp_row_product<S, V, RB, RB>(starts, cols, vals, d_old, row, lane, sbuf, acc);
    size_t base = (size_t)row * RB;
    V rn[RB];
#pragma unroll
    for (int q = 0; q < RB; ++q) rn[q] = r[base + q] - acc[q];
    int p = lane < RB ? lane : 0;
    V z = V(0);
#pragma unroll
    for (int q = 0; q < RB; ++q) z += V(dinv[base * RB + p * RB + q]) * rn[q];
    V dn = keep * d_old[base + p] + step * z;
    V mine = select_lane<V, RB>(rn, p);
    __syncwarp();
    if (lane < RB) {
      r[base + p] = mine;
      d_new[base + p] = dn;
      V xn = x[base + p] + dn;
      if (outer)
        outer[base + p] = outer[base + p] + xn;
      else
        x[base + p] = xn;
    }
  }
}

// The smoother's start from a zero guess (cycle.rs:591-610): r = b; d = (D^-1 b) / theta; x = d.
// B is the type the right-hand side arrives in: f64 at the finest level of an f32 cycle, which
// rounds it here (cycle.rs:236-238) into `b_out`.
template <typename S, typename V, typename B, int RB>
__global__ void __launch_bounds__(kThreads) cheb_start_kernel(uint32_t rows, const S* __restrict__ dinv,
                                                               const B* __restrict__ b_in, V* __restrict__ b_out,
                                                               V* __restrict__ r, V* __restrict__ d,
                                                               V* __restrict__ x, V theta,
                                                               const int* __restrict__ status) {
  if (*status != ST_ACTIVE) return;
  for (uint32_t row = blockIdx.x * blockDim.x + threadIdx.x; row < rows; row += gridDim.x * blockDim.x) {
    size_t base = (size_t)row * RB;
    V bv[RB];
#pragma unroll
    for (int q = 0; q < RB; ++q) {
      bv[q] = V(b_in[base + q]);
      if (b_out) b_out[base + q] = bv[q];
      r[base + q] = bv[q];
    }
#pragma unroll
    for (int p = 0; p < RB; ++p) {
      V z = V(0);
#pragma unroll
      for (int q = 0; q < RB; ++q) z += V(dinv[base * RB + p * RB + q]) * bv[q];
      V dv = z / theta;
      d[base + p] = dv;
      x[base + p] = dv;
    }
  }
}

template <typename V>
__global__ void add_kernel(size_t n, V* __restrict__ x, const V* __restrict__ y, const int* __restrict__ status) {
  if (*status != ST_ACTIVE) return;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    x[i] = x[i] + y[i];
}

// The coarsest level's direct solve as x = V(A^-1 widen(b)), one warp per row of the f64 inverse
// (cycle.rs:476-486 solves with the f64 factor; the inverse is that factor's L^-T L^-1).
template <typename V>
__global__ void __launch_bounds__(kThreads) coarse_solve_kernel(uint32_t n, const double* __restrict__ inv,
                                                                 const V* __restrict__ b, V* __restrict__ x,
                                                                 const int* __restrict__ status) {
  if (*status != ST_ACTIVE) return;
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint32_t row = blockIdx.x * kWarps + warp; row < n; row += gridDim.x * kWarps) {
    const double* a = inv + (size_t)row * n;
    double s = 0.0;
    for (uint32_t j = lane; j < n; j += 32) s += __ldg(a + j) * (double)b[j];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
    if (lane == 0) x[row] = V(s);
  }
}

// ------------------------------------------------------------ fixed-order reductions
__device__ __forceinline__ double block_sum(double v, double* sh) {
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (warp == 0) {
    t = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(kFull, t, o);
  }
  return t;  // valid in warp 0
}

// Each block writes its partials; the last block to finish sums them in block order.
template <int K>
__device__ __forceinline__ bool finish_partials(double (&v)[K], double* partials, unsigned* ticket, double (&total)[K]) {
  __shared__ double sh[32];
  __shared__ bool last;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double s = block_sum(v[k], sh);
    if (threadIdx.x == 0) partials[(size_t)k * gridDim.x + blockIdx.x] = s;
  }
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double s = 0.0;
    for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x) s += __ldcg(partials + (size_t)k * gridDim.x + i);
    total[k] = block_sum(s, sh);
  }
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

// ap = A p on the f64 system with the curvature p.ap; then alpha = rz / curvature
// (pcg.rs:217-228).
__global__ void __launch_bounds__(kThreads) pcg_spmv_dot_kernel(uint32_t rows, const uint32_t* __restrict__ starts,
                                                                 const uint32_t* __restrict__ cols,
                                                                 const double* __restrict__ vals,
                                                                 const double* __restrict__ p, double* __restrict__ ap,
                                                                 double* partials, PcgState* st) {
  if (st->status != ST_ACTIVE) return;
  extern __shared__ int4 smem[];
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int4* sbuf = smem + warp * Slab<double, 3, 3>::kInt4;
  double local = 0.0;
  for (uint32_t row = blockIdx.x * kWarps + warp; row < rows; row += gridDim.x * kWarps) {
    double acc[3];
    warp_row_product<double, double, 3, 3>(starts, cols, vals, p, row, lane, sbuf, acc);
    if (lane < 3) {
      double sum = select_lane<double, 3>(acc, lane);
      size_t i = (size_t)row * 3 + lane;
      ap[i] = sum;
      local += p[i] * sum;
    }
  }
  double v[1] = {local}, total[1];
  if (finish_partials<1>(v, partials, &st->tickets[0], total) && threadIdx.x == 0) {
    double curvature = total[0];
    st->curvature = curvature;
    if (isnan(curvature) || curvature <= 0.0 || !isfinite(st->rz)) {
      st->status = ST_FAILED_NOT_PD;
      st->fail_iteration = st->iterations;
    } else {
      st->alpha = st->rz / curvature;
    }
  }
}

// x += alpha p; r -= alpha ap; relative residual from r.r (pcg.rs:228-234).
__global__ void __launch_bounds__(kThreads) pcg_update_kernel(uint32_t n, const double* __restrict__ p,
                                                               const double* __restrict__ ap, double* __restrict__ x,
                                                               double* __restrict__ r, double* partials, PcgState* st) {
  if (st->status != ST_ACTIVE) return;
  double alpha = st->alpha, na = -alpha;
  double local = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] += alpha * p[i];
    double rv = r[i] + na * ap[i];
    r[i] = rv;
    local += rv * rv;
  }
  double v[1] = {local}, total[1];
  if (finish_partials<1>(v, partials, &st->tickets[1], total) && threadIdx.x == 0) {
    st->iterations += 1;
    double rel = sqrt(total[0]) / st->rhs_norm;
    st->rel = rel;
    st->mode = rel <= st->tolerance ? MODE_CHECK : MODE_NORMAL;
  }
}

// The true residual when the recursive one reports convergence, with the rounding floor of the
// product (pcg.rs:234-255, csr.rs:142-154): r = b - A x; converge, or restart from it.
__global__ void __launch_bounds__(kThreads) pcg_check_kernel(uint32_t rows, const uint32_t* __restrict__ starts,
                                                              const uint32_t* __restrict__ cols,
                                                              const double* __restrict__ vals,
                                                              const double* __restrict__ x, const double* __restrict__ b,
                                                              double* __restrict__ r, double* partials, PcgState* st) {
  if (st->status != ST_ACTIVE || st->mode != MODE_CHECK) return;
  extern __shared__ int4 smem[];
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int4* sbuf = smem + warp * Slab<double, 3, 3>::kInt4;
  double res2 = 0.0, bound2 = 0.0;
  const double eps = 2.220446049250313e-16;
  for (uint32_t row = blockIdx.x * kWarps + warp; row < rows; row += gridDim.x * kWarps) {
    double acc[3];
    warp_row_product<double, double, 3, 3>(starts, cols, vals, x, row, lane, sbuf, acc);
    // |a_ij x_j| row sums for the floor: a second pass over the staged row.
    double mag[3] = {0.0, 0.0, 0.0};
    uint32_t s = starts[row], e = starts[row + 1];
    for (uint32_t at = s + lane; at < e; at += 32) {
      uint32_t c = cols[at];
      const double* blk = vals + (size_t)at * 9;
#pragma unroll
      for (int pp = 0; pp < 3; ++pp)
#pragma unroll
        for (int q = 0; q < 3; ++q) mag[pp] += fabs(blk[pp * 3 + q] * x[(size_t)c * 3 + q]);
    }
#pragma unroll
    for (int pp = 0; pp < 3; ++pp)
      for (int o = 16; o > 0; o >>= 1) mag[pp] += __shfl_xor_sync(kFull, mag[pp], o);
    if (lane < 3) {
      size_t i = (size_t)row * 3 + lane;
      double res = b[i] - select_lane<double, 3>(acc, lane);
      r[i] = res;
      res2 += res * res;
      double bound = (double)((e - s) * 3) * eps * select_lane<double, 3>(mag, lane);
      bound2 += bound * bound;
    }
  }
  double v[2] = {res2, bound2}, total[2];
  if (finish_partials<2>(v, partials, &st->tickets[2], total) && threadIdx.x == 0) {
    double rel = sqrt(total[0]) / st->rhs_norm;
    double floor = sqrt(total[1]) / st->rhs_norm;
    st->rel = rel;
    st->floor = floor;
    st->at_floor = (rel > st->tolerance && rel <= floor) ? 1 : 0;
    if (rel <= st->tolerance || st->at_floor)
      st->status = ST_CONVERGED;
    else
      st->mode = MODE_RESTART;
  }
}

// rz' = r.z and beta (pcg.rs:257-263): Fletcher-Reeves rz'/rz, or in flexible mode
// (z'.(r' - r))/rz with r' - r = -alpha ap. A restart takes p = z (pcg.rs:278-282). Then the
// iteration cap (pcg.rs:266-273).
template <typename Z>
__global__ void __launch_bounds__(kThreads) pcg_dot_rz_kernel(uint32_t n, const double* __restrict__ r,
                                                               const Z* __restrict__ z, const double* __restrict__ ap,
                                                               double* partials, PcgState* st) {
  if (st->status != ST_ACTIVE) return;
  bool flex = st->flexible && st->mode == MODE_NORMAL;
  double rz = 0.0, apz = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double zv = (double)z[i];
    rz += r[i] * zv;
    if (flex) apz += ap[i] * zv;
  }
  double v[2] = {rz, apz}, total[2];
  if (finish_partials<2>(v, partials, &st->tickets[3], total) && threadIdx.x == 0) {
    double rz_next = total[0];
    if (st->mode == MODE_RESTART) {
      st->beta = 0.0;
    } else if (st->flexible) {
      st->beta = (-st->alpha * total[1]) / st->rz;
    } else {
      st->beta = rz_next / st->rz;
    }
    st->rz = rz_next;
    if (st->iterations >= st->max_iterations) st->status = ST_FAILED_NOT_CONVERGED;
  }
}

// p = z + beta p, or p = z after a restart.
template <typename Z>
__global__ void pcg_update_p_kernel(uint32_t n, const Z* __restrict__ z, double* __restrict__ p, PcgState* st) {
  if (st->status != ST_ACTIVE) return;
  bool restart = st->mode == MODE_RESTART;
  double beta = st->beta;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double zv = (double)z[i];
    p[i] = restart ? zv : zv + beta * p[i];
  }
}

// Initial state (Pcg::new, pcg.rs:135-164): x = 0, r = b, rhs norm; then reset_direction.
__global__ void __launch_bounds__(kThreads) pcg_init_kernel(uint32_t n, const double* __restrict__ b, double* __restrict__ x,
                                                             double* __restrict__ r, double* partials, PcgState* st) {
  double local = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] = 0.0;
    r[i] = b[i];
    local += b[i] * b[i];
  }
  double v[1] = {local}, total[1];
  if (finish_partials<1>(v, partials, &st->tickets[4], total) && threadIdx.x == 0) {
    st->rhs_norm = sqrt(total[0]);
    st->rel = 1.0;
    st->mode = MODE_RESTART;
    st->status = st->rhs_norm == 0.0 ? ST_CONVERGED : ST_ACTIVE;
    if (st->rhs_norm == 0.0) st->rel = 0.0;
  }
}

// Jacobi: z = r / diag (preconditioner.rs:237-247), stored as the inverse diagonal.
__global__ void jacobi_kernel(uint32_t n, const double* __restrict__ inv, const double* __restrict__ r,
                              double* __restrict__ z, const int* __restrict__ status) {
  if (*status != ST_ACTIVE) return;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) z[i] = r[i] * inv[i];
}

// ------------------------------------------------------------ launch helpers
int g_sm_count = 0;

int grid_for_rows(size_t rows_per_unit_work) {
  if (g_sm_count == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (g_sm_count <= 0) g_sm_count = 148;
  }
  size_t blocks = (rows_per_unit_work + kWarps - 1) / kWarps;
  size_t cap = (size_t)g_sm_count * 8;
  return (int)std::max<size_t>(1, std::min(blocks, cap));
}

int grid_for_elems(size_t n) {
  size_t blocks = (n + kThreads - 1) / kThreads;
  size_t cap = (size_t)(g_sm_count ? g_sm_count : 148) * 8;
  return (int)std::max<size_t>(1, std::min(blocks, cap));
}

template <typename K>
void smem_opt_in(K kernel, int bytes) {
  if (bytes > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

template <typename S, typename V, int RB, int CB, int OP>
void launch_bsr(const DevBsr& m, const V* x, V* y, const V* b, const int* status, cudaStream_t st) {
  int smem = kWarps * Slab<S, RB, CB>::kInt4 * 16;
  auto k = bsr_kernel<S, V, RB, CB, OP>;
  static bool opted = false;
  if (!opted) {
    smem_opt_in(k, smem);
    opted = true;
  }
  k<<<grid_for_rows(m.rows), kThreads, smem, st>>>(m.rows, m.starts, m.cols, (const S*)m.vals, x, y, b, status);
}

template <typename S, typename V, int RB, int OP>
void bsr_dispatch_cb(const DevBsr& m, const V* x, V* y, const V* b, const int* status, cudaStream_t st) {
  if (m.cb == 3)
    launch_bsr<S, V, RB, 3, OP>(m, x, y, b, status, st);
  else
    launch_bsr<S, V, RB, 6, OP>(m, x, y, b, status, st);
}

template <typename S, typename V, int OP>
void bsr_dispatch(const DevBsr& m, const V* x, V* y, const V* b, const int* status, cudaStream_t st) {
  if (m.rb == 3)
    bsr_dispatch_cb<S, V, 3, OP>(m, x, y, b, status, st);
  else
    bsr_dispatch_cb<S, V, 6, OP>(m, x, y, b, status, st);
}

template <typename S, typename V, int RB>
void launch_cheb_step(const DevLevel& L, const V* d_old, V* d_new, V* r, V* x, V* outer, double keep, double step,
                      const int* status, cudaStream_t st) {
  int smem = kWarps * Slab<S, RB, RB>::kInt4 * 16;
  auto k = cheb_step_kernel<S, V, RB>;
  static bool opted = false;
  if (!opted) {
    smem_opt_in(k, smem);
    opted = true;
  }
  k<<<grid_for_rows(L.a.rows), kThreads, smem, st>>>(L.a.rows, L.a.starts, L.a.cols, (const S*)L.a.vals,
                                                     (const S*)L.dinv, d_old, d_new, r, x, outer, (V)keep, (V)step,
                                                     status);
}

template <typename S, typename V, typename B, int RB>
void launch_cheb_start(const DevLevel& L, const B* b_in, V* b_out, V* r, V* d, V* x, double theta, const int* status,
                       cudaStream_t st) {
  cheb_start_kernel<S, V, B, RB><<<grid_for_elems(L.a.rows), kThreads, 0, st>>>(
      L.a.rows, (const S*)L.dinv, b_in, b_out, r, d, x, (V)theta, status);
}

// The smoother from a zero guess on right-hand side b into x (cycle.rs:570-651). `outer`, when
// given, receives x += (smoothed x) at the last step instead of storing x.
template <typename S, typename V, typename B>
void enqueue_smooth(DeviceSolver& s, DevLevel& L, const B* b_in, V* b_out, V* x, V* outer, const int* status) {
  cudaStream_t st = s.stream;
  V* r = (V*)L.res;
  V* d[2] = {(V*)L.d0, (V*)L.d1};
  if (L.a.rb == 3)
    launch_cheb_start<S, V, B, 3>(L, b_in, b_out, r, d[0], x, L.theta, status, st);
  else
    launch_cheb_start<S, V, B, 6>(L, b_in, b_out, r, d[0], x, L.theta, status, st);
  s.launches_per_iteration++;
  for (size_t k = 0; k < L.steps.size(); ++k) {
    bool last = k + 1 == L.steps.size();
    V* o = last ? outer : nullptr;
    if (L.a.rb == 3)
      launch_cheb_step<S, V, 3>(L, d[k & 1], d[(k + 1) & 1], r, x, o, L.steps[k].first, L.steps[k].second, status, st);
    else
      launch_cheb_step<S, V, 6>(L, d[k & 1], d[(k + 1) & 1], r, x, o, L.steps[k].first, L.steps[k].second, status, st);
    s.launches_per_iteration++;
  }
  if (outer && L.steps.empty()) {
    add_kernel<V><<<grid_for_elems(L.n), kThreads, 0, st>>>(L.n, outer, x, status);
    s.launches_per_iteration++;
  }
}

// One V-cycle from level `li` (cycle.rs:461-539). B is the type of the right-hand side.
template <typename S, typename V, typename B>
void enqueue_cycle(DeviceSolver& s, size_t li, const B* rhs, V* b_store, V* x, const int* status) {
  DevLevel& L = s.levels[li];
  cudaStream_t st = s.stream;
  // The level's right-hand side in V: rounded into b_store when it arrives as another type.
  if (!L.has_p) {
    if (L.has_factor) {
      const V* bv = (const V*)rhs;
      if (b_store) {
        // An f64 right-hand side reaching an f32 coarsest level directly (a one-level hierarchy).
        enqueue_smooth<S, V, B>(s, L, rhs, b_store, (V*)L.tmp, nullptr, status);
        bv = b_store;
      }
      coarse_solve_kernel<V><<<grid_for_rows(L.n), kThreads, 0, st>>>(L.n, L.coarse_inverse, bv, x, status);
      s.launches_per_iteration++;
    } else {
      enqueue_smooth<S, V, B>(s, L, rhs, b_store, x, nullptr, status);
    }
    return;
  }
  enqueue_smooth<S, V, B>(s, L, rhs, b_store, x, nullptr, status);
  const V* b = b_store ? (const V*)b_store : (const V*)rhs;
  DevLevel& C = s.levels[li + 1];
  bsr_dispatch<S, V, OP_RESIDUAL>(L.a, x, (V*)L.res, b, status, st);
  bsr_dispatch<S, V, OP_SET>(L.r, (const V*)L.res, (V*)C.b, nullptr, status, st);
  s.launches_per_iteration += 2;
  enqueue_cycle<S, V, V>(s, li + 1, (const V*)C.b, nullptr, (V*)C.x, status);
  bsr_dispatch<S, V, OP_ADD>(L.p, (const V*)C.x, x, nullptr, status, st);
  bsr_dispatch<S, V, OP_RESIDUAL>(L.a, x, (V*)L.tmp, b, status, st);
  s.launches_per_iteration += 2;
  enqueue_smooth<S, V, V>(s, L, (const V*)L.tmp, nullptr, (V*)L.post_x, x, status);
}

// z = M r for the solver's r (f64) into z (f64) or z32.
void enqueue_precondition(DeviceSolver& s, const double* r, double* z, float* z32, const int* status) {
  if (!s.multigrid) {
    jacobi_kernel<<<grid_for_elems(s.n), kThreads, 0, s.stream>>>(s.n, s.jacobi, r, z, status);
    s.launches_per_iteration++;
    return;
  }
  DevLevel& L0 = s.levels[0];
  if (!s.storage_single)
    enqueue_cycle<double, double, double>(s, 0, r, nullptr, z, status);
  else if (!s.vector_single)
    enqueue_cycle<float, double, double>(s, 0, r, nullptr, z, status);
  else
    enqueue_cycle<float, float, double>(s, 0, r, (float*)L0.b, z32, status);
}

}  // namespace

sf_status cuda_check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return SF_OK;
  char msg[200];
  std::snprintf(msg, sizeof(msg), "%s: %s", what, cudaGetErrorString(e));
  if (e == cudaErrorMemoryAllocation) return fail(SF_DEVICE_MEMORY_BUDGET, msg);
  return fail(SF_CUDA_ERROR, msg);
}

sf_status dev_alloc(DeviceSolver& s, void** ptr, size_t bytes) {
  // 64 bytes of slack: the staged loads read whole 16-byte chunks past an array's last value.
  size_t padded = bytes + 64;
  cudaError_t e = cudaMalloc(ptr, padded);
  if (e != cudaSuccess) return cuda_check(e, "cudaMalloc");
  cudaMemsetAsync(*ptr, 0, padded, s.stream);
  s.owned.push_back(*ptr);
  s.bytes += padded;
  return SF_OK;
}

void dev_free_all(DeviceSolver& s) {
  if (s.graph_exec) cudaGraphExecDestroy(s.graph_exec);
  if (s.graph) cudaGraphDestroy(s.graph);
  s.graph_exec = nullptr;
  s.graph = nullptr;
  for (void* p : s.owned) cudaFree(p);
  s.owned.clear();
  s.bytes = 0;
}

namespace {

template <typename S>
sf_status upload_bsr(DeviceSolver& s, const Bsr& h, DevBsr& d) {
  d.rows = (uint32_t)h.rows;
  d.rb = (uint32_t)h.rb;
  d.cb = (uint32_t)h.cb;
  d.blocks = h.cols.size();
  if (sf_status e = dev_alloc(s, (void**)&d.starts, (h.rows + 1) * 4)) return e;
  if (sf_status e = dev_alloc(s, (void**)&d.cols, std::max<size_t>(1, h.cols.size()) * 4)) return e;
  if (sf_status e = dev_alloc(s, &d.vals, std::max<size_t>(1, h.vals.size()) * sizeof(S))) return e;
  copy_h2d(s, d.starts, h.starts.data(), (h.rows + 1) * 4);
  if (!h.cols.empty()) copy_h2d(s, d.cols, h.cols.data(), h.cols.size() * 4);
  if (!h.vals.empty()) {
    if (sizeof(S) == 8) {
      copy_h2d(s, d.vals, h.vals.data(), h.vals.size() * 8);
    } else {
      std::vector<float> f(h.vals.size());
      for (size_t i = 0; i < f.size(); ++i) f[i] = (float)h.vals[i];
      copy_h2d(s, d.vals, f.data(), f.size() * 4);
      cudaStreamSynchronize(s.stream);
    }
  }
  return cuda_check(cudaGetLastError(), "upload");
}

// The explicit transpose of a prolongator: coarse rows, fine block columns ascending, blocks
// transposed (gpu/layout.rs:254-291 stores the same for gather restriction).
Bsr transpose(const Bsr& p, size_t coarse_rows) {
  Bsr t;
  t.rows = coarse_rows;
  t.rb = p.cb;
  t.cb = p.rb;
  t.starts.assign(coarse_rows + 1, 0);
  for (uint32_t c : p.cols) t.starts[c + 1] += 1;
  for (size_t i = 0; i < coarse_rows; ++i) t.starts[i + 1] += t.starts[i];
  std::vector<uint32_t> fill(t.starts.begin(), t.starts.end() - 1);
  t.cols.resize(p.cols.size());
  t.vals.resize(p.vals.size());
  size_t len = p.rb * p.cb;
  for (size_t row = 0; row < p.rows; ++row)
    for (uint32_t at = p.starts[row]; at < p.starts[row + 1]; ++at) {
      uint32_t c = p.cols[at];
      uint32_t o = fill[c]++;
      t.cols[o] = (uint32_t)row;
      for (size_t a = 0; a < p.rb; ++a)
        for (size_t b = 0; b < p.cb; ++b) t.vals[(size_t)o * len + b * p.rb + a] = p.vals[(size_t)at * len + a * p.cb + b];
    }
  return t;
}

}  // namespace

sf_status solver_upload_hierarchy(DeviceSolver& s, const std::vector<HostLevel>& levels, uint64_t degree) {
  size_t S = s.storage_single ? 4 : 8, V = s.vector_single ? 4 : 8;
  s.levels.assign(levels.size(), DevLevel());
  for (size_t li = 0; li < levels.size(); ++li) {
    const HostLevel& h = levels[li];
    DevLevel& L = s.levels[li];
    L.n = (uint32_t)(h.a.rows * h.a.rb);
    if (li == 0 && !s.storage_single) {
      L.a = s.system;  // the f64 system matrix is the finest operator
    } else {
      sf_status e = s.storage_single ? upload_bsr<float>(s, h.a, L.a) : upload_bsr<double>(s, h.a, L.a);
      if (e) return e;
    }
    if (sf_status e = dev_alloc(s, &L.dinv, h.inverse_diagonal.size() * S)) return e;
    if (S == 8) {
      copy_h2d(s, L.dinv, h.inverse_diagonal.data(), h.inverse_diagonal.size() * 8);
    } else {
      std::vector<float> f(h.inverse_diagonal.begin(), h.inverse_diagonal.end());
      copy_h2d(s, L.dinv, f.data(), f.size() * 4);
      cudaStreamSynchronize(s.stream);
    }
    L.has_p = h.has_p;
    if (h.has_p) {
      Bsr t = transpose(h.p, levels[li + 1].a.rows);
      sf_status e = s.storage_single ? upload_bsr<float>(s, h.p, L.p) : upload_bsr<double>(s, h.p, L.p);
      if (e) return e;
      e = s.storage_single ? upload_bsr<float>(s, t, L.r) : upload_bsr<double>(s, t, L.r);
      if (e) return e;
    }
    L.has_factor = h.has_factor;
    if (h.has_factor) {
      if (sf_status e = dev_alloc(s, (void**)&L.coarse_inverse, h.coarse_inverse.size() * 8)) return e;
      copy_h2d(s, L.coarse_inverse, h.coarse_inverse.data(), h.coarse_inverse.size() * 8);
    }
    // ChebyshevCoefficients (gpu/layout.rs:443-465), the recurrence of cycle.rs:578-626.
    double theta = 0.5 * (h.lambda_max + h.lambda_min);
    double delta = 0.5 * (h.lambda_max - h.lambda_min);
    double sigma = theta / delta;
    double rho = 1.0 / sigma;
    L.theta = theta;
    L.steps.clear();
    for (uint64_t k = 1; k < degree; ++k) {
      double next = 1.0 / (2.0 * sigma - rho);
      L.steps.push_back({next * rho, 2.0 * next / delta});
      rho = next;
    }
    void** vecs[] = {&L.b, &L.x, &L.res, &L.z, &L.d0, &L.d1, &L.post_x, &L.tmp};
    for (void** v : vecs)
      if (sf_status e = dev_alloc(s, v, (size_t)L.n * V)) return e;
  }
  if (s.vector_single)
    if (sf_status e = dev_alloc(s, (void**)&s.z32, (size_t)s.n * 4)) return e;
  return cuda_check(cudaStreamSynchronize(s.stream), "hierarchy upload");
}

sf_status solver_init_pcg(DeviceSolver& s, double tolerance, uint64_t max_iterations) {
  PcgState h;
  std::memset(&h, 0, sizeof(h));
  h.tolerance = tolerance;
  h.max_iterations = max_iterations ? max_iterations : 10ull * s.n + 1000ull;
  h.flexible = s.flexible ? 1 : 0;
  h.status = ST_ACTIVE;
  copy_h2d(s, s.state, &h, sizeof(h));
  int one_active = ST_ACTIVE;
  copy_h2d(s, s.always_active, &one_active, sizeof(int));
  pcg_init_kernel<<<kReduceBlocks, kReduceThreads, 0, s.stream>>>(s.n, s.rhs, s.x, s.r, s.partials, s.state);
  return solver_enqueue_reset(s);
}

sf_status solver_enqueue_reset(DeviceSolver& s) {
  const int* status = &s.state->status;
  enqueue_precondition(s, s.r, s.z, s.z32, status);
  if (s.vector_single && s.multigrid) {
    pcg_dot_rz_kernel<float><<<kReduceBlocks, kReduceThreads, 0, s.stream>>>(s.n, s.r, s.z32, s.ap, s.partials, s.state);
    pcg_update_p_kernel<float><<<grid_for_elems(s.n), kThreads, 0, s.stream>>>(s.n, s.z32, s.p, s.state);
  } else {
    pcg_dot_rz_kernel<double><<<kReduceBlocks, kReduceThreads, 0, s.stream>>>(s.n, s.r, s.z, s.ap, s.partials, s.state);
    pcg_update_p_kernel<double><<<grid_for_elems(s.n), kThreads, 0, s.stream>>>(s.n, s.z, s.p, s.state);
  }
  return cuda_check(cudaGetLastError(), "reset direction");
}

sf_status solver_enqueue_iteration(DeviceSolver& s) {
  cudaStream_t st = s.stream;
  const int* status = &s.state->status;
  s.launches_per_iteration = 0;
  int smem = kWarps * Slab<double, 3, 3>::kInt4 * 16;
  pcg_spmv_dot_kernel<<<kReduceBlocks, kThreads, smem, st>>>(s.system.rows, s.system.starts, s.system.cols,
                                                             (const double*)s.system.vals, s.p, s.ap, s.partials,
                                                             s.state);
  pcg_update_kernel<<<kReduceBlocks, kReduceThreads, 0, st>>>(s.n, s.p, s.ap, s.x, s.r, s.partials, s.state);
  pcg_check_kernel<<<kReduceBlocks, kThreads, smem, st>>>(s.system.rows, s.system.starts, s.system.cols,
                                                          (const double*)s.system.vals, s.x, s.rhs, s.r, s.partials,
                                                          s.state);
  s.launches_per_iteration += 3;
  enqueue_precondition(s, s.r, s.z, s.z32, status);
  if (s.vector_single && s.multigrid) {
    pcg_dot_rz_kernel<float><<<kReduceBlocks, kReduceThreads, 0, st>>>(s.n, s.r, s.z32, s.ap, s.partials, s.state);
    pcg_update_p_kernel<float><<<grid_for_elems(s.n), kThreads, 0, st>>>(s.n, s.z32, s.p, s.state);
  } else {
    pcg_dot_rz_kernel<double><<<kReduceBlocks, kReduceThreads, 0, st>>>(s.n, s.r, s.z, s.ap, s.partials, s.state);
    pcg_update_p_kernel<double><<<grid_for_elems(s.n), kThreads, 0, st>>>(s.n, s.z, s.p, s.state);
  }
  s.launches_per_iteration += 2;
  return cuda_check(cudaGetLastError(), "iteration");
}

sf_status solver_capture_graph(DeviceSolver& s) {
  if (s.graph_exec) return SF_OK;
  cudaError_t e = cudaStreamBeginCapture(s.stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return cuda_check(e, "begin capture");
  sf_status st = solver_enqueue_iteration(s);
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(s.stream, &g);
  if (st) return st;
  if (e != cudaSuccess) return cuda_check(e, "end capture");
  s.graph = g;
  size_t nodes = 0;
  cudaGraphGetNodes(g, nullptr, &nodes);
  s.graph_kernels = nodes;
  e = cudaGraphInstantiate(&s.graph_exec, g, 0);
  return cuda_check(e, "graph instantiate");
}

sf_status solver_restart(DeviceSolver& s, double tolerance, uint64_t max_iterations) {
  s.launches_per_iteration = 0;
  sf_status e = solver_init_pcg(s, tolerance, max_iterations);
  s.launches += s.launches_per_iteration + 1;
  return e;
}

namespace {

template <typename S, typename V>
sf_status time_level0(DeviceSolver& s, int kernel, uint64_t repeats, double* ms, double* bytes) {
  DevLevel& L = s.levels[0];
  const int* on = s.always_active;
  double rows = L.a.rows, blocks = (double)L.a.blocks, rb = L.a.rb, sv = sizeof(V), ss = sizeof(S);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, s.stream);
  for (uint64_t i = 0; i < repeats; ++i) {
    if (kernel == SF_KERNEL_CHEBYSHEV_STEP) {
      V* d[2] = {(V*)L.d0, (V*)L.d1};
      launch_cheb_step<S, V, 3>(L, d[i & 1], d[(i + 1) & 1], (V*)L.res, (V*)L.x, nullptr, 0.5, 0.25, on, s.stream);
    } else if (kernel == SF_KERNEL_LEVEL_RESIDUAL) {
      launch_bsr<S, V, 3, 3, OP_RESIDUAL>(L.a, (const V*)L.x, (V*)L.tmp, (const V*)L.b, on, s.stream);
    } else {
      bsr_dispatch<S, V, OP_SET>(L.r, (const V*)L.res, (V*)s.levels[1].b, nullptr, on, s.stream);
    }
  }
  cudaEventRecord(b, s.stream);
  cudaError_t e = cudaEventSynchronize(b);
  float t = 0;
  cudaEventElapsedTime(&t, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *ms = t / (double)repeats;
  double matrix = rows * 4 + blocks * (rb * rb * ss + 4);
  double vec = rows * rb * sv;
  if (kernel == SF_KERNEL_CHEBYSHEV_STEP)
    *bytes = matrix + vec /* d_old */ + 2 * vec /* r */ + rows * rb * rb * ss /* D^-1 */ + vec /* d_new */ + 2 * vec /* x */;
  else if (kernel == SF_KERNEL_LEVEL_RESIDUAL)
    *bytes = matrix + 3 * vec;
  else
    *bytes = (double)L.r.rows * 4 + (double)L.r.blocks * (L.r.rb * L.r.cb * ss + 4) + vec +
             (double)L.r.rows * L.r.rb * sv;
  s.launches += repeats;
  return cuda_check(e, "time kernel");
}

}  // namespace

sf_status solver_time_kernel(DeviceSolver& s, int kernel, uint64_t repeats, double* ms, double* bytes) {
  if (repeats == 0) return fail(SF_INVALID_ARGUMENT, "repeats must be positive");
  if (kernel == SF_KERNEL_SYSTEM_PRODUCT) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, s.stream);
    for (uint64_t i = 0; i < repeats; ++i)
      launch_bsr<double, double, 3, 3, OP_SET>(s.system, s.p, s.ap, nullptr, s.always_active, s.stream);
    cudaEventRecord(b, s.stream);
    cudaError_t e = cudaEventSynchronize(b);
    float t = 0;
    cudaEventElapsedTime(&t, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *ms = t / (double)repeats;
    *bytes = (double)s.system.rows * 4 + (double)s.system.blocks * 76 + (double)s.n * 16;
    s.launches += repeats;
    return cuda_check(e, "time kernel");
  }
  if (!s.multigrid || s.levels.empty()) return fail(SF_INVALID_ARGUMENT, "the study has no multigrid hierarchy");
  if (kernel == SF_KERNEL_RESTRICTION && !s.levels[0].has_p) return fail(SF_INVALID_ARGUMENT, "one-level hierarchy");
  if (kernel < 0 || kernel > SF_KERNEL_RESTRICTION) return fail(SF_INVALID_ARGUMENT, "unknown kernel");
  if (!s.storage_single) return time_level0<double, double>(s, kernel, repeats, ms, bytes);
  if (!s.vector_single) return time_level0<float, double>(s, kernel, repeats, ms, bytes);
  return time_level0<float, float>(s, kernel, repeats, ms, bytes);
}

sf_status solver_precondition(DeviceSolver& s, const double* d_in, double* d_out) {
  enqueue_precondition(s, d_in, d_out, s.z32, s.always_active);
  if (s.vector_single && s.multigrid) {
    // widen the f32 correction
    std::vector<float> h(s.n);
    copy_d2h(s, h.data(), s.z32, (size_t)s.n * 4);
    cudaStreamSynchronize(s.stream);
    std::vector<double> w(h.begin(), h.end());
    copy_h2d(s, d_out, w.data(), (size_t)s.n * 8);
  }
  return cuda_check(cudaStreamSynchronize(s.stream), "precondition");
}

sf_status solver_system_multiply(DeviceSolver& s, const double* d_in, double* d_out) {
  launch_bsr<double, double, 3, 3, OP_SET>(s.system, d_in, d_out, nullptr, s.always_active, s.stream);
  return cuda_check(cudaStreamSynchronize(s.stream), "system multiply");
}

sf_status solver_read_state(DeviceSolver& s, PcgState* out) {
  copy_d2h(s, out, s.state, sizeof(PcgState));
  return cuda_check(cudaStreamSynchronize(s.stream), "read state");
}

}  // namespace sf
