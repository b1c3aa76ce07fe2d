// The solve path on sm_100a: the block-CSR products of the V-cycle and the conjugate gradient,
// the fused Chebyshev smoother, restriction through the stored transpose, prolongation, the
// coarsest level's dense solve and the FP64 conjugate gradient with fixed-order reductions.
//
// The block products are HBM-bound streams over each operator's value slab. A matrix's rows are
// cut on the host into row groups (consecutive rows, about 4 KB of values each). A warp walks its
// groups in a grid-stride loop and stages each one into its own shared-memory buffer with 16-byte
// cp.async copies (L2 only), double-buffered: while it multiplies group k out of shared memory,
// group k+1 is already streaming in, so every warp keeps kilobytes in flight without register
// cost. A row is shared by `LPR` lanes (32 for the stiffness and transpose operators, fewer for
// the thin prolongators), each multiplying one block at a time with its x gathered through L2;
// the lanes' sums meet in a fixed xor butterfly, so every run gives the same bits. Each kernel
// reads the solver's status word first and returns at once when the solve has ended, so a batch
// of iterations can be enqueued (or replayed as a CUDA graph) without a host round trip each.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <cstring>
#include <cstdlib>
#include <utility>

#include "device.h"

namespace sf {

namespace {

const unsigned kFull = 0xffffffffu;
const int kThreads = 256;
const int kWarps = kThreads / 32;
const uint32_t kGroupTarget = 4096;     // value bytes a row group aims at
const int kSmemPerBlockTarget = 72 * 1024;

// ------------------------------------------------------------ programmatic dependent launch
// Every solve kernel is launched with programmatic stream serialization: its launch is prepared
// while the predecessor runs, and at entry it waits until the predecessor grid has completed and
// its writes are visible (griddepcontrol.wait). The data dependence is unchanged; without a
// programmatic predecessor the wait returns at once.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
}


// ------------------------------------------------------------ kernel bodies and batched launches
// Every solve kernel is written as a __device__ body. A launch either runs it as a single-instance
// grid (its arguments by value) or, while a recorder is active, records the arguments so that a
// batch of instances with the same launch sequence can run each step as ONE grid: blockIdx.y
// selects the instance, whose arguments (operator, vectors, Chebyshev scalars, status word) come
// from a device table. The status word of each instance is its convergence mask: a finished
// instance's blocks return at once.
template <typename... P>
struct Pack;
template <>
struct Pack<> {};
template <typename H, typename... T>
struct Pack<H, T...> {
  H head;
  Pack<T...> tail;
};

inline Pack<> make_pack() { return {}; }
template <typename H, typename... T>
Pack<H, T...> make_pack(H h, T... t) {
  Pack<H, T...> p;
  p.head = h;
  p.tail = make_pack(t...);
  return p;
}

template <auto Body, typename... Done>
__device__ __forceinline__ void apply_pack(const Pack<>&, Done... done) {
  Body(done...);
}
template <auto Body, typename H, typename... T, typename... Done>
__device__ __forceinline__ void apply_pack(const Pack<H, T...>& p, Done... done) {
  apply_pack<Body>(p.tail, done..., p.head);
}

template <auto Body, typename... P>
__global__ void __launch_bounds__(kThreads) single_kernel(P... args) {
  pdl_enter();
  Body(args...);
}
template <auto Body, typename PackT>
__global__ void __launch_bounds__(kThreads) batched_kernel(const PackT* __restrict__ table) {
  pdl_enter();
  const PackT a = table[blockIdx.y];
  apply_pack<Body>(a);
}

// The same wrappers for a body launched with `Threads` threads per block (the coarse tail).
template <auto Body, int Threads, typename... P>
__global__ void __launch_bounds__(Threads) single_kernel_n(P... args) {
  pdl_enter();
  Body(args...);
}
template <auto Body, int Threads, typename PackT>
__global__ void __launch_bounds__(Threads) batched_kernel_n(const PackT* __restrict__ table) {
  pdl_enter();
  const PackT a = table[blockIdx.y];
  apply_pack<Body>(a);
}

template <typename F>
struct BodyTraits;
template <typename... P>
struct BodyTraits<void (*)(P...)> {
  typedef Pack<P...> PackT;
  template <typename... A>
  static PackT pack(A&&... a) {
    return make_pack<P...>(static_cast<P>(a)...);
  }
  template <auto Body>
  static const void* single() {
    return (const void*)single_kernel<Body, P...>;
  }
  template <auto Body>
  static const void* batched() {
    return (const void*)batched_kernel<Body, PackT>;
  }
  template <auto Body, int Threads>
  static const void* single_n() {
    return (const void*)single_kernel_n<Body, Threads, P...>;
  }
  template <auto Body, int Threads>
  static const void* batched_n() {
    return (const void*)batched_kernel_n<Body, Threads, PackT>;
  }
};

}  // namespace

thread_local std::vector<LaunchRecord>* g_recorder = nullptr;

namespace {

inline void fill_argv(void**, Pack<>&) {}
template <typename H, typename... T>
void fill_argv(void** out, Pack<H, T...>& p) {
  out[0] = &p.head;
  fill_argv(out + 1, p.tail);
}

template <auto Body, typename... A>
void launch_body(dim3 grid, dim3 block, size_t smem, cudaStream_t st, A&&... args) {
  typedef BodyTraits<decltype(Body)> T;
  typename T::PackT pk = T::pack(std::forward<A>(args)...);
  if (g_recorder) {
    LaunchRecord r;
    r.batched = T::template batched<Body>();
    r.grid = grid;
    r.block = block;
    r.smem = smem;
    r.pack.resize(sizeof(pk));
    std::memcpy(r.pack.data(), &pk, sizeof(pk));
    g_recorder->push_back(std::move(r));
    return;
  }
  const void* k = T::template single<Body>();
  if (smem > 48 * 1024) {
    // The opt-in above 48 KB is a per-device attribute of the kernel: set it once per device
    // ordinal (a bit per device, atomically, since studies on different host threads and devices
    // launch the same kernels).
    static std::atomic<uint64_t> opted{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const uint64_t bit = dev < 64 ? 1ull << dev : 0;
    if (!bit || !(opted.load(std::memory_order_acquire) & bit)) {
      cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
      opted.fetch_or(bit, std::memory_order_acq_rel);
    }
  }
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  void* argv[sizeof...(A) + 1];
  fill_argv(argv, pk);
  cudaLaunchKernelExC(&cfg, k, argv);
}

// A launch of `grid.x` CTAs of Threads threads forming one thread-block cluster per grid row (no
// programmatic serialization: the launch waits for its predecessor in stream order).
template <auto Body, int Threads, typename... A>
void launch_body_cluster(dim3 grid, size_t smem, cudaStream_t st, A&&... args) {
  typedef BodyTraits<decltype(Body)> T;
  typename T::PackT pk = T::pack(std::forward<A>(args)...);
  const dim3 block(Threads);
  if (g_recorder) {
    LaunchRecord r;
    r.batched = T::template batched_n<Body, Threads>();
    r.grid = grid;
    r.block = block;
    r.smem = smem;
    r.cluster = grid.x;
    r.pack.resize(sizeof(pk));
    std::memcpy(r.pack.data(), &pk, sizeof(pk));
    g_recorder->push_back(std::move(r));
    return;
  }
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = grid.x;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  void* argv[sizeof...(A) + 1];
  fill_argv(argv, pk);
  cudaLaunchKernelExC(&cfg, T::template single_n<Body, Threads>(), argv);
}

// ------------------------------------------------------------ asynchronous staging
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Issues the copies of [src, src + bytes) into dst as whole aligned 16-byte chunks; returns the
// byte offset of src inside dst. The chunks may reach 15 bytes past either end of the range:
// every device array is allocated 256-byte aligned with 64 bytes of slack at its end.
__device__ __forceinline__ int stage_async(const void* src, uint32_t bytes, char* dst, int lane) {
  uintptr_t a = reinterpret_cast<uintptr_t>(src);
  uintptr_t a0 = a & ~uintptr_t(15);
  int off = (int)(a - a0);
  int chunks = (int)((off + bytes + 15) >> 4);
  const char* g = reinterpret_cast<const char*>(a0);
  for (int c = lane; c < chunks; c += 32) cp_async16(dst + 16 * c, g + 16 * c);
  return off;
}

// A block matrix as the kernels read it. Each row group is described by {first row, end row,
// first block, end block}, so a warp needs one 16-byte load to start staging a group.
template <typename S>
struct Op {
  const uint32_t* __restrict__ starts;
  const uint32_t* __restrict__ cols;
  const S* __restrict__ vals;
  const uint4* __restrict__ groups;
  uint32_t ngroups;
  uint32_t vbuf, cbuf, sbuf;  // bytes of one value / column / row-start staging buffer
};

template <typename S>
Op<S> op_of(const DevBsr& m) {
  Op<S> o;
  o.starts = m.starts;
  o.cols = m.cols;
  o.vals = (const S*)m.vals;
  o.groups = m.groups;
  o.ngroups = m.ngroups;
  o.vbuf = (m.group_bytes + 31) & ~15u;
  o.cbuf = (m.group_blocks * 4 + 31) & ~15u;
  o.sbuf = ((m.group_rows + 1) * 4 + 31) & ~15u;
  return o;
}

template <typename S>
__host__ __device__ __forceinline__ uint32_t slot_bytes(const Op<S>& A) {
  return A.vbuf + A.cbuf + A.sbuf;
}

// Gates: the row walks (run_groups, sell_rows, split_rows) test their kernel's gate (the status
// word) only after their first operator loads have been requested, so the status load and those
// loads travel together instead of one after the other. The operator arrays are never written by
// a solve kernel, and a closed gate ends the walk before any x gather, epilogue load or store.
// sell_rows' and split_rows' row-map loads are volatile so the compiler keeps them ahead of the
// gate's branch.
__device__ __forceinline__ uint32_t ld_early(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.global.nc.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

// load() reads the gate's word(s); open() tests them. run_groups issues the load before its first
// operator loads and tests it after them; gate() does both at once.
struct StatusGate {
  const int* status;
  __device__ __forceinline__ int load() const { return *status; }
  __device__ __forceinline__ static bool open(int w) { return w == ST_ACTIVE; }
  __device__ __forceinline__ bool operator()() const { return open(load()); }
};
struct OpenGate {
  __device__ __forceinline__ int load() const { return 0; }
  __device__ __forceinline__ static bool open(int) { return true; }
  __device__ __forceinline__ bool operator()() const { return true; }
};

// The true-residual check runs only in its mode.
struct CheckGate {
  const PcgState* st;
  __device__ __forceinline__ int2 load() const { return make_int2(st->status, st->mode); }
  __device__ __forceinline__ static bool open(int2 w) { return w.x == ST_ACTIVE && w.y == MODE_CHECK; }
  __device__ __forceinline__ bool operator()() const { return open(load()); }
};

// Walks this warp's row groups. Per row (one team of LPR lanes each) it calls epi.pre(row, live,
// lane) before the row's blocks are read, so the epilogue's own loads overlap the gathers, and
// epi.post(row, live, sums[RB], mag[RB], lane) after the team's fixed butterfly, in every lane.
// With MAG it also sums |a_ij x_j| per row (the rounding floor of pcg.rs:246-248). A group is
// staged one grid-stride step ahead (double buffer), its descriptor two steps ahead.
// Returns the gate (uniform over the grid: a body may still reduce across its blocks after true).
template <typename S, typename V, int RB, int CB, int LPR, bool MAG, class Epi, class Gate>
__device__ __forceinline__ bool run_groups(const Op<S>& A, const V* __restrict__ x, char* wbase, Epi& epi,
                                           const Gate& gate) {
  constexpr int LEN = RB * CB;
  constexpr int TEAMS = 32 / LPR;
  const int lane = threadIdx.x & 31;
  const int team = lane / LPR, tl = lane % LPR;
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  uint32_t g = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const uint32_t sb = slot_bytes(A);
  int vo0 = 0, vo1 = 0, co0 = 0, co1 = 0, so0 = 0, so1 = 0;
  auto issue = [&](const uint4& d, int slot) {
    char* base = wbase + slot * sb;
    int vo = stage_async(A.vals + (size_t)d.z * LEN, (d.w - d.z) * LEN * (uint32_t)sizeof(S), base, lane);
    int co = stage_async(A.cols + d.z, (d.w - d.z) * 4u, base + A.vbuf, lane);
    int so = stage_async(A.starts + d.x, (d.y - d.x + 1) * 4u, base + A.vbuf + A.cbuf, lane);
    if (slot) {
      vo1 = vo;
      co1 = co;
      so1 = so;
    } else {
      vo0 = vo;
      co0 = co;
      so0 = so;
    }
  };
  const uint4 none = make_uint4(0, 0, 0, 0);
  // The gate's load goes first (the staging asm below is a compiler memory barrier) and is tested
  // once the first group's staging is in flight; a closed gate drains the copies and ends.
  const auto word = gate.load();
  uint4 cur = g < A.ngroups ? A.groups[g] : none;
  uint4 nxt = g + nw < A.ngroups ? A.groups[g + nw] : none;
  if (g < A.ngroups) issue(cur, 0);
  cp_async_commit();
  if (!Gate::open(word)) {
    cp_async_wait_all();
    return false;
  }
  for (int k = 0; g < A.ngroups; ++k, g += nw) {
    const int slot = k & 1;
    const bool has_next = g + nw < A.ngroups;
    if (has_next) issue(nxt, slot ^ 1);
    uint4 after = g + 2 * nw < A.ngroups ? A.groups[g + 2 * nw] : none;
    cp_async_commit();
    cp_async_wait_one();
    __syncwarp();
    char* base = wbase + slot * sb;
    const S* vals = reinterpret_cast<const S*>(base + (slot ? vo1 : vo0));
    const uint32_t* cols = reinterpret_cast<const uint32_t*>(base + A.vbuf + (slot ? co1 : co0));
    const uint32_t* rst = reinterpret_cast<const uint32_t*>(base + A.vbuf + A.cbuf + (slot ? so1 : so0));
    const uint32_t nrows = cur.y - cur.x;
    for (uint32_t rb = 0; rb < nrows; rb += TEAMS) {
      const uint32_t lr = rb + team;
      const bool live = lr < nrows;
      const uint32_t row = cur.x + (live ? lr : 0);
      epi.pre(row, live, tl);
      V acc[RB], mag[RB];
#pragma unroll
      for (int p = 0; p < RB; ++p) acc[p] = mag[p] = V(0);
      if (live) {
        const uint32_t b0 = rst[lr] - cur.z, b1 = rst[lr + 1] - cur.z;
        for (uint32_t j = b0 + tl; j < b1; j += 2 * LPR) {
          const uint32_t j2 = j + LPR;
          const bool two = j2 < b1;
          const uint32_t c0 = cols[j], c1 = two ? cols[j2] : c0;
          V xa[CB], xb[CB];
#pragma unroll
          for (int q = 0; q < CB; ++q) {
            xa[q] = __ldg(x + (size_t)c0 * CB + q);
            xb[q] = __ldg(x + (size_t)c1 * CB + q);
          }
          const S* ba = vals + (size_t)j * LEN;
          const S* bb = vals + (size_t)(two ? j2 : j) * LEN;
#pragma unroll
          for (int p = 0; p < RB; ++p)
#pragma unroll
            for (int q = 0; q < CB; ++q) {
              V t = V(ba[p * CB + q]) * xa[q];
              acc[p] += t;
              if (MAG) mag[p] += fabs(t);
            }
          if (two) {
#pragma unroll
            for (int p = 0; p < RB; ++p)
#pragma unroll
              for (int q = 0; q < CB; ++q) {
                V t = V(bb[p * CB + q]) * xb[q];
                acc[p] += t;
                if (MAG) mag[p] += fabs(t);
              }
          }
        }
      }
      __syncwarp();
#pragma unroll
      for (int p = 0; p < RB; ++p)
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) {
          acc[p] += __shfl_xor_sync(kFull, acc[p], o);
          if (MAG) mag[p] += __shfl_xor_sync(kFull, mag[p], o);
        }
      epi.post(row, live, acc, mag, tl);
    }
    __syncwarp();
    cur = nxt;
    nxt = after;
  }
  cp_async_wait_all();
  return true;
}

template <typename V, int RB>
__device__ __forceinline__ V pick(const V (&v)[RB], int p) {
  V out = v[0];
#pragma unroll
  for (int q = 1; q < RB; ++q)
    if (p == q) out = v[q];
  return out;
}

// The components p = lane, lane + LPR, ... < RB of a row this lane finishes.
template <int RB, int LPR>
struct Parts {
  static constexpr int N = (RB + LPR - 1) / LPR;
};

enum { OP_SET = 0, OP_RESIDUAL = 1, OP_ADD = 2 };

// y = A x, y = b - A x, or y = y + A x.
template <typename V, int RB, int LPR, int OP>
struct EpiAxpy {
  V* __restrict__ y;
  const V* __restrict__ b;
  V in[Parts<RB, LPR>::N];
  __device__ __forceinline__ void pre(uint32_t row, bool live, int tl) {
    if (OP == OP_SET || !live) return;
#pragma unroll
    for (int k = 0; k < Parts<RB, LPR>::N; ++k) {
      int p = tl + k * LPR;
      if (p < RB) in[k] = OP == OP_RESIDUAL ? b[(size_t)row * RB + p] : y[(size_t)row * RB + p];
    }
  }
  __device__ __forceinline__ void post(uint32_t row, bool live, const V (&acc)[RB], const V (&)[RB], int tl) {
    if (!live) return;
#pragma unroll
    for (int k = 0; k < Parts<RB, LPR>::N; ++k) {
      int p = tl + k * LPR;
      if (p >= RB) continue;
      size_t i = (size_t)row * RB + p;
      V sum = pick<V, RB>(acc, p);
      if (OP == OP_SET) y[i] = sum;
      if (OP == OP_RESIDUAL) y[i] = in[k] - sum;
      if (OP == OP_ADD) y[i] = in[k] + sum;
    }
  }
};

template <typename S, typename V, int RB, int CB, int LPR, int OP>
__device__ __forceinline__ void bsr_kernel(Op<S> A, const V* __restrict__ x, V* __restrict__ y,
                                                       const V* __restrict__ b, const int* __restrict__ status) {
  extern __shared__ __align__(16) char smem[];
  char* wbase = smem + (threadIdx.x >> 5) * 2 * slot_bytes(A);
  EpiAxpy<V, RB, LPR, OP> epi{y, b, {}};
  run_groups<S, V, RB, CB, LPR, false>(A, x, wbase, epi, StatusGate{status});
}

// One Chebyshev step fused with its product (cycle.rs:611-650): ad = A d_old; r -= ad;
// z = D^-1 r; d_new = keep d_old + step z; x += d_new. With `outer` set (the last step of the
// post-smoother) the smoothed correction goes straight into the level's x: outer += (x + d_new),
// the reference's post_x += d and then x += post_x (cycle.rs:533-536).
template <typename S, typename V, int RB, int LPR>
struct EpiCheb {
  static constexpr int N = Parts<RB, LPR>::N;
  const S* __restrict__ dinv;
  const V* __restrict__ d_old;
  V* __restrict__ d_new;
  V* __restrict__ r;
  V* __restrict__ x;
  V* __restrict__ outer;
  V keep, step;
  V rv[RB];
  V dv[N], xv[N], ov[N];
  S di[N][RB];
  __device__ __forceinline__ void pre(uint32_t row, bool live, int tl) {
    if (!live) return;
    const size_t base = (size_t)row * RB;
#pragma unroll
    for (int q = 0; q < RB; ++q) rv[q] = r[base + q];
#pragma unroll
    for (int k = 0; k < N; ++k) {
      int p = tl + k * LPR;
      if (p >= RB) continue;
#pragma unroll
      for (int q = 0; q < RB; ++q) di[k][q] = dinv[base * RB + p * RB + q];
      dv[k] = d_old[base + p];
      xv[k] = x[base + p];
      if (outer) ov[k] = outer[base + p];
    }
  }
  __device__ __forceinline__ void post(uint32_t row, bool live, const V (&acc)[RB], const V (&)[RB], int tl) {
    if (!live) return;
    const size_t base = (size_t)row * RB;
    V rn[RB];
#pragma unroll
    for (int q = 0; q < RB; ++q) rn[q] = rv[q] - acc[q];
#pragma unroll
    for (int k = 0; k < N; ++k) {
      int p = tl + k * LPR;
      if (p >= RB) continue;
      V z = V(0);
#pragma unroll
      for (int q = 0; q < RB; ++q) z += V(di[k][q]) * rn[q];
      V dn = keep * dv[k] + step * z;
      r[base + p] = pick<V, RB>(rn, p);
      d_new[base + p] = dn;
      V xn = xv[k] + dn;
      if (outer)
        outer[base + p] = ov[k] + xn;
      else
        x[base + p] = xn;
    }
  }
};

template <typename S, typename V, int RB, int LPR>
__device__ __forceinline__ void cheb_step_kernel(Op<S> A, const S* __restrict__ dinv, const V* __restrict__ d_old,
                                                             V* __restrict__ d_new, V* __restrict__ r, V* __restrict__ x,
                                                             V* __restrict__ outer, V keep, V step,
                                                             const int* __restrict__ status) {
  extern __shared__ __align__(16) char smem[];
  char* wbase = smem + (threadIdx.x >> 5) * 2 * slot_bytes(A);
  EpiCheb<S, V, RB, LPR> epi;
  epi.dinv = dinv;
  epi.d_old = d_old;
  epi.d_new = d_new;
  epi.r = r;
  epi.x = x;
  epi.outer = outer;
  epi.keep = keep;
  epi.step = step;
  run_groups<S, V, RB, RB, LPR, false>(A, d_old, wbase, epi, StatusGate{status});
}

// The smoother's start from a zero guess (cycle.rs:591-610): r = b; d = (D^-1 b) / theta; x = d.
// B is the type the right-hand side arrives in: f64 at the finest level of an f32 cycle, which
// rounds it here (cycle.rs:236-238) into `b_out`.
template <typename S, typename V, typename B, int RB>
__device__ __forceinline__ void cheb_start_kernel(uint32_t rows, const S* __restrict__ dinv,
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
__device__ __forceinline__ void add_kernel(size_t n, V* __restrict__ x, const V* __restrict__ y, const int* __restrict__ status) {
  if (*status != ST_ACTIVE) return;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    x[i] = x[i] + y[i];
}

template <typename B, typename V>
__device__ __forceinline__ void convert_kernel(size_t n, const B* __restrict__ in, V* __restrict__ out, const int* __restrict__ status) {
  if (*status != ST_ACTIVE) return;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = V(in[i]);
}

// The coarsest level's direct solve as x = V(A^-1 widen(b)), one warp per row of the f64 inverse
// (cycle.rs:476-486 solves with the f64 factor; the inverse is that factor's L^-T L^-1).
template <typename V>
__device__ __forceinline__ void coarse_solve_kernel(uint32_t n, const double* __restrict__ inv,
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
// The conjugate gradient's vector kernels walk [0, n) with a grid stride. A thread loads the
// elements of kStrides consecutive strides before it uses any of them (one round trip to memory
// instead of kStrides dependent ones) and then sums them in stride order: the same order, and so
// the same bits, as the plain loop.
constexpr int kStrides = 4;
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

// ------------------------------------------------------------ SELL-32: one thread per row
// For operators with many rows (the finest level and the f64 system): a warp holds a slice of 32
// rows of similar length, each thread sums its own row's blocks in column order. A thread reads
// its row in chunks of 144 bytes of values (nine 16-byte vector loads, each 512 contiguous bytes
// across the warp) plus one vector load of the chunk's columns. No shared memory, no shuffles:
// the instruction stream is the blocks' FMAs plus their loads.
template <typename S>
struct SellOp {
  const uint32_t* __restrict__ rows;
  const uint32_t* __restrict__ len;
  const uint32_t* __restrict__ start;
  const uint32_t* __restrict__ cols;
  const S* __restrict__ vals;
  uint32_t nslices, nrows;
};

template <typename S>
SellOp<S> sell_of(const DevBsr& m) {
  SellOp<S> o;
  o.rows = m.sell_rows;
  o.len = m.sell_len;
  o.start = m.sell_start;
  o.cols = m.sell_cols;
  o.vals = (const S*)m.sell_vals;
  o.nslices = m.nslices;
  o.nrows = m.rows;
  return o;
}

template <typename S>
struct Vec16;
template <>
struct Vec16<float> {
  typedef float4 type;
  __device__ __forceinline__ static void split(const float4& w, float* out) {
    out[0] = w.x;
    out[1] = w.y;
    out[2] = w.z;
    out[3] = w.w;
  }
};
template <>
struct Vec16<double> {
  typedef double2 type;
  __device__ __forceinline__ static void split(const double2& w, double* out) {
    out[0] = w.x;
    out[1] = w.y;
  }
};

template <int U>
__device__ __forceinline__ void load_cols(const uint32_t* p, uint32_t (&c)[U]) {
  if constexpr (U == 4) {
    uint4 w = __ldcs(reinterpret_cast<const uint4*>(p));
    c[0] = w.x;
    c[1] = w.y;
    c[2] = w.z;
    c[3] = w.w;
  } else if constexpr (U == 2) {
    uint2 w = __ldcs(reinterpret_cast<const uint2*>(p));
    c[0] = w.x;
    c[1] = w.y;
  } else {
#pragma unroll
    for (int u = 0; u < U; ++u) c[u] = __ldcs(p + u);
  }
}

// Returns the gate: false when the kernel must end (uniform over the grid, so a body may still
// reduce across its blocks after a true return).
template <typename S, typename V, int RB, int CB, bool MAG, class Epi, class Gate>
__device__ __forceinline__ bool sell_rows(const SellOp<S>& A, const V* __restrict__ x, Epi& epi, const Gate& gate) {
  constexpr int LEN = RB * CB;
  constexpr int U = sell_chunk_blocks(LEN, (int)sizeof(S));
  constexpr int VEC = 16 / (int)sizeof(S);
  constexpr int NV = U * LEN / VEC;
  static_assert((U * LEN) % VEC == 0, "a lane chunk is whole 16-byte vectors");
  typedef typename Vec16<S>::type W;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = blockDim.x >> 5;
  bool open = false;
  for (uint32_t s = blockIdx.x * warps + (threadIdx.x >> 5); s < A.nslices; s += gridDim.x * warps) {
    const uint32_t slot = s * 32 + lane;
    const uint32_t row = ld_early(A.rows + slot);
    const uint32_t n = ld_early(A.len + slot);
    const uint32_t base = ld_early(A.start + s);
    if (!open) {
      if (!gate()) return false;
      open = true;
    }
    const bool live = row < A.nrows;
    epi.pre(row, live);
    V acc[RB], mag[RB];
#pragma unroll
    for (int p = 0; p < RB; ++p) acc[p] = mag[p] = V(0);
    // One chunk of U blocks per step: its columns in one vector load, its values in NV 16-byte
    // vector loads (each a contiguous 512 bytes across the warp). The values of chunk k+1 are
    // issued before chunk k's x gathers and FMAs, so a chunk's stream latency hides behind the
    // previous chunk's gathers; the columns run one chunk further ahead (chunk k+2), so the x
    // gathers of a chunk never wait on the DRAM load of its own columns. The FMAs run in column
    // order, so the row's sum keeps its sequential order.
    uint32_t cn[U], cf[U];
    S vn[U * LEN];
    if (n > 0) {
      load_cols<U>(A.cols + base + lane * U, cn);
      const W* vp = reinterpret_cast<const W*>(A.vals + (size_t)base * LEN) + lane;
#pragma unroll
      for (int q = 0; q < NV; ++q) Vec16<S>::split(__ldcs(vp + 32 * q), vn + q * VEC);
    }
    if (U < n) load_cols<U>(A.cols + base + 32 * U + lane * U, cf);
    for (uint32_t k0 = 0; k0 < n; k0 += U) {
      uint32_t c[U];
      S v[U * LEN];
#pragma unroll
      for (int u = 0; u < U; ++u) c[u] = cn[u];
#pragma unroll
      for (int i = 0; i < U * LEN; ++i) v[i] = vn[i];
      if (k0 + U < n) {
        const uint32_t q1 = base + 32 * (k0 + U);
#pragma unroll
        for (int u = 0; u < U; ++u) cn[u] = cf[u];
        const W* vp = reinterpret_cast<const W*>(A.vals + (size_t)q1 * LEN) + lane;
#pragma unroll
        for (int q = 0; q < NV; ++q) Vec16<S>::split(__ldcs(vp + 32 * q), vn + q * VEC);
        if (k0 + 2 * U < n) load_cols<U>(A.cols + q1 + 32 * U + lane * U, cf);
      }
      V xv[U][CB];
#pragma unroll
      for (int u = 0; u < U; ++u)
#pragma unroll
        for (int q = 0; q < CB; ++q) xv[u][q] = k0 + u < n ? __ldg(x + (size_t)c[u] * CB + q) : V(0);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (k0 + u >= n) break;
#pragma unroll
        for (int p = 0; p < RB; ++p)
#pragma unroll
          for (int q = 0; q < CB; ++q) {
            V t = V(v[u * LEN + p * CB + q]) * xv[u][q];
            acc[p] += t;
            if (MAG) mag[p] += fabs(t);
          }
      }
    }
    epi.post(row, live, n, acc, mag);
  }
  return open || gate();
}

template <typename V, int RB, int OP>
struct SellAxpy {
  V* __restrict__ y;
  const V* __restrict__ b;
  V in[RB];
  __device__ __forceinline__ void pre(uint32_t row, bool live) {
    if (OP == OP_SET || !live) return;
#pragma unroll
    for (int p = 0; p < RB; ++p) in[p] = OP == OP_RESIDUAL ? b[(size_t)row * RB + p] : y[(size_t)row * RB + p];
  }
  __device__ __forceinline__ void post(uint32_t row, bool live, uint32_t, const V (&acc)[RB], const V (&)[RB]) {
    if (!live) return;
#pragma unroll
    for (int p = 0; p < RB; ++p) {
      size_t i = (size_t)row * RB + p;
      if (OP == OP_SET) y[i] = acc[p];
      if (OP == OP_RESIDUAL) y[i] = in[p] - acc[p];
      if (OP == OP_ADD) y[i] = in[p] + acc[p];
    }
  }
};

template <typename S, typename V, int RB, int CB, int OP>
__device__ __forceinline__ void sell_kernel(SellOp<S> A, const V* __restrict__ x, V* __restrict__ y,
                                                        const V* __restrict__ b, const int* __restrict__ status) {
  SellAxpy<V, RB, OP> epi{y, b, {}};
  sell_rows<S, V, RB, CB, false>(A, x, epi, StatusGate{status});
}

// The fused Chebyshev step of cheb_step_kernel, one thread per row.
template <typename S, typename V, int RB>
struct SellCheb {
  const S* __restrict__ dinv;
  const V* __restrict__ d_old;
  V* __restrict__ d_new;
  V* __restrict__ r;
  V* __restrict__ x;
  V* __restrict__ outer;
  V keep, step;
  // The row's own operands are loaded after its blocks: every thread already keeps several
  // blocks' loads in flight, and holding these 21 values across the block loop would cost the
  // registers of a resident block.
  __device__ __forceinline__ void pre(uint32_t, bool) {}
  __device__ __forceinline__ void post(uint32_t row, bool live, uint32_t, const V (&acc)[RB], const V (&)[RB]) {
    if (!live) return;
    const size_t base = (size_t)row * RB;
    V rn[RB];
#pragma unroll
    for (int q = 0; q < RB; ++q) rn[q] = r[base + q] - acc[q];
#pragma unroll
    for (int p = 0; p < RB; ++p) {
      V z = V(0);
#pragma unroll
      for (int q = 0; q < RB; ++q) z += V(dinv[base * RB + p * RB + q]) * rn[q];
      V dn = keep * d_old[base + p] + step * z;
      r[base + p] = rn[p];
      d_new[base + p] = dn;
      V xn = x[base + p] + dn;
      if (outer)
        outer[base + p] = outer[base + p] + xn;
      else
        x[base + p] = xn;
    }
  }
};

template <typename S, typename V, int RB>
__device__ __forceinline__ void sell_cheb_kernel(SellOp<S> A, const S* __restrict__ dinv,
                                                             const V* __restrict__ d_old, V* __restrict__ d_new,
                                                             V* __restrict__ r, V* __restrict__ x, V* __restrict__ outer,
                                                             V keep, V step, const int* __restrict__ status) {
  SellCheb<S, V, RB> epi;
  epi.dinv = dinv;
  epi.d_old = d_old;
  epi.d_new = d_new;
  epi.r = r;
  epi.x = x;
  epi.outer = outer;
  epi.keep = keep;
  epi.step = step;
  sell_rows<S, V, RB, RB, false>(A, d_old, epi, StatusGate{status});
}

// ------------------------------------------------------------ split rows: one thread per scalar row
// For operators of 6-row blocks with many block rows (level 1, and the transpose restricting onto
// it): one lane per scalar row gives six times the threads of SELL-32 and a chain of chunks one
// sixth as long per thread, with no shared memory. Lane t = 6 m + p of a slice owns scalar row p
// of the slice's block row m; the six lanes of a block row read its shared column chunk (one
// address per block row) and gather the same x entries. Each block's cb products are summed in
// column order, a chunk's block sums pairwise, and the chunk sums in column order: a row of an
// f32 level is summed about as accurately as the row-group engine's lane sums and butterfly
// (a plain running sum over the row's ~100 products left the f32 cycle visibly noisier).
template <int U>
__device__ __forceinline__ void load_cols_shared(const uint32_t* p, uint32_t (&c)[U]) {
  if constexpr (U % 4 == 0) {
#pragma unroll
    for (int k = 0; k < U / 4; ++k) {
      uint4 w = __ldg(reinterpret_cast<const uint4*>(p) + k);
      c[4 * k] = w.x;
      c[4 * k + 1] = w.y;
      c[4 * k + 2] = w.z;
      c[4 * k + 3] = w.w;
    }
  } else if constexpr (U % 2 == 0) {
#pragma unroll
    for (int k = 0; k < U / 2; ++k) {
      uint2 w = __ldg(reinterpret_cast<const uint2*>(p) + k);
      c[2 * k] = w.x;
      c[2 * k + 1] = w.y;
    }
  } else {
#pragma unroll
    for (int u = 0; u < U; ++u) c[u] = __ldg(p + u);
  }
}

template <typename S, typename V, int CB, class Epi, class Gate>
__device__ __forceinline__ bool split_rows(const SellOp<S>& A, const V* __restrict__ x, Epi& epi, const Gate& gate) {
  constexpr int U = sell_chunk_blocks(CB, (int)sizeof(S));
  constexpr int VEC = 16 / (int)sizeof(S);
  constexpr int NV = U * CB / VEC;
  static_assert((U * CB) % VEC == 0, "a lane chunk is whole 16-byte vectors");
  typedef typename Vec16<S>::type W;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t m = lane / 6, part = lane - 6 * m;
  const uint32_t warps = blockDim.x >> 5;
  bool open = false;  // the gate, tested after the first slice's row map is requested (sell_rows)
  for (uint32_t s = blockIdx.x * warps + (threadIdx.x >> 5); s < A.nslices; s += gridDim.x * warps) {
    const uint32_t slot = s * 32 + lane;
    const uint32_t row = ld_early(A.rows + slot);
    const uint32_t n = ld_early(A.len + slot);
    const uint32_t base = ld_early(A.start + s);
    if (!open) {
      if (!gate()) return false;
      open = true;
    }
    const bool live = row < A.nrows;
    epi.pre(row, part, live);
    V acc = V(0);
    const uint32_t* cp = A.cols + (size_t)(base >> 5) * kSplitRowsPerSlice + (size_t)m * U;
    // Values one chunk ahead, columns two (as in sell_rows).
    uint32_t cn[U], cf[U];
    S vn[U * CB];
    if (n > 0) {
      load_cols_shared<U>(cp, cn);
      const W* vp = reinterpret_cast<const W*>(A.vals + (size_t)base * CB) + lane;
#pragma unroll
      for (int q = 0; q < NV; ++q) Vec16<S>::split(__ldcs(vp + 32 * q), vn + q * VEC);
    }
    if (U < n) load_cols_shared<U>(cp + (size_t)kSplitRowsPerSlice * U, cf);
    for (uint32_t k0 = 0; k0 < n; k0 += U) {
      uint32_t c[U];
      S v[U * CB];
#pragma unroll
      for (int u = 0; u < U; ++u) c[u] = cn[u];
#pragma unroll
      for (int i = 0; i < U * CB; ++i) v[i] = vn[i];
      if (k0 + U < n) {
#pragma unroll
        for (int u = 0; u < U; ++u) cn[u] = cf[u];
        const W* vp = reinterpret_cast<const W*>(A.vals + ((size_t)base + 32 * (k0 + U)) * CB) + lane;
#pragma unroll
        for (int q = 0; q < NV; ++q) Vec16<S>::split(__ldcs(vp + 32 * q), vn + q * VEC);
        if (k0 + 2 * U < n) load_cols_shared<U>(cp + (size_t)kSplitRowsPerSlice * (k0 + 2 * U), cf);
      }
      V xv[U][CB];
#pragma unroll
      for (int u = 0; u < U; ++u)
#pragma unroll
        for (int q = 0; q < CB; ++q) xv[u][q] = k0 + u < n ? __ldg(x + (size_t)c[u] * CB + q) : V(0);
      V bs[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        bs[u] = V(v[u * CB]) * xv[u][0];
#pragma unroll
        for (int q = 1; q < CB; ++q) bs[u] += V(v[u * CB + q]) * xv[u][q];
      }
#pragma unroll
      for (int w = 1; w < U; w *= 2)
#pragma unroll
        for (int u = 0; u + w < U; u += 2 * w) bs[u] += bs[u + w];
      acc += bs[0];
    }
    epi.post(row, part, live, acc);
  }
  return open || gate();
}

template <typename V, int OP>
struct SplitAxpy {
  V* __restrict__ y;
  const V* __restrict__ b;
  V in;
  __device__ __forceinline__ void pre(uint32_t row, uint32_t part, bool live) {
    if (OP == OP_SET || !live) return;
    const size_t i = (size_t)row * 6 + part;
    in = OP == OP_RESIDUAL ? b[i] : y[i];
  }
  __device__ __forceinline__ void post(uint32_t row, uint32_t part, bool live, V acc) {
    if (!live) return;
    const size_t i = (size_t)row * 6 + part;
    if (OP == OP_SET) y[i] = acc;
    if (OP == OP_RESIDUAL) y[i] = in - acc;
    if (OP == OP_ADD) y[i] = in + acc;
  }
};

template <typename S, typename V, int CB, int OP>
__device__ __forceinline__ void split_kernel(SellOp<S> A, const V* __restrict__ x, V* __restrict__ y,
                                             const V* __restrict__ b, const int* __restrict__ status) {
  SplitAxpy<V, OP> epi{y, b, V(0)};
  split_rows<S, V, CB>(A, x, epi, StatusGate{status});
}

// The fused Chebyshev step with split rows. z = D^-1 r couples a block row's six components:
// each lane's new residual reaches the other five lanes of its block row by shuffles (every
// lane of the warp takes part; idle lanes carry zeros), then lane p forms row p of D^-1 r in
// the order of cheb_step_kernel.
template <typename S, typename V>
struct SplitCheb {
  const S* __restrict__ dinv;
  const V* __restrict__ d_old;
  V* __restrict__ d_new;
  V* __restrict__ r;
  V* __restrict__ x;
  V* __restrict__ outer;
  V keep, step;
  __device__ __forceinline__ void pre(uint32_t, uint32_t, bool) {}
  __device__ __forceinline__ void post(uint32_t row, uint32_t part, bool live, V acc) {
    const size_t i = (size_t)row * 6 + part;
    const V rn = live ? r[i] - acc : V(0);
    const uint32_t first = (threadIdx.x & 31) - part;
    V rq[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) rq[q] = __shfl_sync(kFull, rn, (first + q) & 31);
    if (!live) return;
    V z = V(0);
#pragma unroll
    for (int q = 0; q < 6; ++q) z += V(dinv[i * 6 + q]) * rq[q];
    const V dn = keep * d_old[i] + step * z;
    r[i] = rn;
    d_new[i] = dn;
    const V xn = x[i] + dn;
    if (outer)
      outer[i] = outer[i] + xn;
    else
      x[i] = xn;
  }
};

template <typename S, typename V>
__device__ __forceinline__ void split_cheb_kernel(SellOp<S> A, const S* __restrict__ dinv,
                                                  const V* __restrict__ d_old, V* __restrict__ d_new,
                                                  V* __restrict__ r, V* __restrict__ x, V* __restrict__ outer,
                                                  V keep, V step, const int* __restrict__ status) {
  SplitCheb<S, V> epi;
  epi.dinv = dinv;
  epi.d_old = d_old;
  epi.d_new = d_new;
  epi.r = r;
  epi.x = x;
  epi.outer = outer;
  epi.keep = keep;
  epi.step = step;
  split_rows<S, V, 6>(A, d_old, epi, StatusGate{status});
}

// ------------------------------------------------------------ the coarse tail: one cluster launch
// The last smoothed level s and the coarsest level's direct solve run as ONE launch of one
// thread-block cluster per instance (cycle.rs:461-539 for levels s and s + 1): smoother start,
// Chebyshev steps, residual, restriction, coarse solve, prolongation, residual and post-smoother
// are phases whose rows are split over the cluster's CTAs, which meet at the hardware cluster
// barrier between phases (arrive.release / wait.acquire at cluster scope; no spin loop of ours).
// A level this small runs each per-phase launch as a few waves of short warps, so the launches,
// not the bytes, set its time. Each CTA stages its share of the rows (operator, prolongator,
// restriction, D^-1, coarse inverse) in shared memory once; the vectors that phases gather live
// as a replica in every CTA, and a phase stores each result into all replicas through distributed
// shared memory, so a phase reads nothing but shared memory. Products use the row-group engine's
// lanes per row, loop order and butterfly, and the epilogues restate EpiAxpy / EpiCheb /
// cheb_start_kernel / coarse_solve_kernel term for term: the tail returns the bits of the
// per-phase launches it replaces. Only the level's final x goes back to global memory.
// Opt-in (sf_study_options.coarse_tail): measured on the 606k-DOF plate, the cluster launch takes
// 44 us against about 37 us for the overlapped per-phase launches; its phases stall on
// instruction fetch and on the cluster barriers rather than on memory.
constexpr int kTailMaxSteps = 4;
// Threads per CTA: 512 for f32 vectors, 256 for f64 (twice the registers per value).
template <typename V>
constexpr int tail_threads() {
  return sizeof(V) == 4 ? 512 : 256;
}
constexpr uint32_t kTailMaxRows = 768;     // block rows of the fused level: a few rows per warp
constexpr uint32_t kTailMaxCoarse = 1024;  // scalar rows of the coarsest level
constexpr size_t kTailMaxSmem = 200 * 1024;

__device__ __forceinline__ void cluster_barrier() {
  __syncwarp();  // the barrier's .aligned form wants the warp converged
  asm volatile("barrier.cluster.arrive.release.aligned;\n"
               "barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

template <typename S>
struct TailMat {
  const uint32_t* __restrict__ starts;
  const uint32_t* __restrict__ cols;
  const S* __restrict__ vals;
  uint32_t rows;
  int lanes;  // lanes per row of the operator's row-group launch
};

template <typename S, typename V>
struct TailArgs {
  TailMat<S> a, r, p;
  const S* dinv;
  const double* inv;  // coarsest level: n x n f64 inverse
  uint32_t nc;
  uint32_t nsteps;
  V theta;
  V keep[kTailMaxSteps], step[kTailMaxSteps];
  const V* b;
  V* x;
  const int* status;
};

// The rows of a phase that CTA i of n takes: [share(rows, n, i), share(rows, n, i + 1)).
__host__ __device__ inline uint32_t tail_share(uint32_t rows, uint32_t n, uint32_t i) {
  return (uint32_t)(((uint64_t)rows * i) / n);
}
__host__ __device__ inline size_t tail_align(size_t bytes) { return (bytes + 15) & ~size_t(15); }

// Shared memory the staged rows of one operator take (starts, columns, 6 x 6 blocks).
__host__ __device__ inline size_t tail_mat_bytes(uint32_t rows, uint32_t blocks, size_t value_bytes) {
  return tail_align((size_t)(rows + 1) * 4) + tail_align((size_t)blocks * 4) + tail_align((size_t)blocks * 36 * value_bytes);
}

// Rows [row0, row0 + rows) of an operator staged in this CTA's shared memory (starts from 0).
template <typename S>
struct LocalMat {
  const uint32_t* starts;
  const uint32_t* cols;
  const S* vals;
  uint32_t row0, rows;
};

// Copies n 16-byte words to shared memory, eight loads in flight per thread before any store.
__device__ __forceinline__ void stage16(float4* __restrict__ dst, const float4* __restrict__ src, size_t n) {
  for (size_t i0 = threadIdx.x; i0 < n; i0 += 8 * (size_t)blockDim.x) {
    float4 w[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const size_t i = i0 + (size_t)k * blockDim.x;
      if (i < n) w[k] = __ldg(src + i);
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const size_t i = i0 + (size_t)k * blockDim.x;
      if (i < n) dst[i] = w[k];
    }
  }
}

template <typename S>
__device__ __forceinline__ LocalMat<S> tail_stage(const TailMat<S>& A, uint32_t r0, uint32_t r1, unsigned char*& at) {
  const uint32_t b0 = A.starts[r0], b1 = A.starts[r1];
  uint32_t* st = reinterpret_cast<uint32_t*>(at);
  at += tail_align((size_t)(r1 - r0 + 1) * 4);
  uint32_t* cl = reinterpret_cast<uint32_t*>(at);
  at += tail_align((size_t)(b1 - b0) * 4);
  S* vl = reinterpret_cast<S*>(at);
  at += tail_align((size_t)(b1 - b0) * 36 * sizeof(S));
  for (uint32_t i = threadIdx.x; i <= r1 - r0; i += blockDim.x) st[i] = A.starts[r0 + i] - b0;
  for (uint32_t i = threadIdx.x; i < b1 - b0; i += blockDim.x) cl[i] = __ldg(A.cols + b0 + i);
  stage16(reinterpret_cast<float4*>(vl), reinterpret_cast<const float4*>(A.vals + (size_t)b0 * 36),
          (size_t)(b1 - b0) * 36 * sizeof(S) / 16);
  LocalMat<S> m;
  m.starts = st;
  m.cols = cl;
  m.vals = vl;
  m.row0 = r0;
  m.rows = r1 - r0;
  return m;
}

// Row p of a staged 6 x 6 block: 24 bytes (f32, 8-byte aligned) or 48 bytes (f64, 16-byte aligned).
__device__ __forceinline__ void block_row(const float* src, float (&v)[6]) {
  const float2* w = reinterpret_cast<const float2*>(src);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    float2 t = w[i];
    v[2 * i] = t.x;
    v[2 * i + 1] = t.y;
  }
}
__device__ __forceinline__ void block_row(const double* src, double (&v)[6]) {
  const double2* w = reinterpret_cast<const double2*>(src);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double2 t = w[i];
    v[2 * i] = t.x;
    v[2 * i + 1] = t.y;
  }
}

// One operator product over this CTA's staged rows with LPR lanes per row (run_groups' order: a
// lane sums its blocks j, j + LPR, j + 2 LPR, ... then the team's butterfly). A block is read one
// row at a time from shared memory, so only six values are live; x is this CTA's replica.
template <typename S, typename V, int LPR, class Epi>
__device__ __forceinline__ void tail_rows(const LocalMat<S>& A, const V* x, Epi& epi) {
  constexpr int RB = 6, CB = 6, LEN = 36;
  constexpr int TEAMS = 32 / LPR;
  const int lane = threadIdx.x & 31;
  const int team = lane / LPR, tl = lane % LPR;
  const uint32_t warps = blockDim.x >> 5;
  for (uint32_t l0 = (threadIdx.x >> 5) * TEAMS; l0 < A.rows; l0 += warps * TEAMS) {
    const uint32_t lr = l0 + team;
    const bool live = lr < A.rows;
    const uint32_t row = A.row0 + lr;
    epi.pre(row, live, tl);
    V acc[RB];
#pragma unroll
    for (int p = 0; p < RB; ++p) acc[p] = V(0);
    if (live) {
      const uint32_t b0 = A.starts[lr], b1 = A.starts[lr + 1];
      for (uint32_t j = b0 + tl; j < b1; j += LPR) {
        const uint32_t c = A.cols[j];
        V xa[CB];
#pragma unroll
        for (int q = 0; q < CB; ++q) xa[q] = x[(size_t)c * CB + q];
        const S* blk = A.vals + (size_t)j * LEN;
#pragma unroll
        for (int p = 0; p < RB; ++p) {
          S v[6];
          block_row(blk + p * CB, v);
#pragma unroll
          for (int q = 0; q < CB; ++q) {
            V t = V(v[q]) * xa[q];
            acc[p] += t;
          }
        }
      }
    }
    __syncwarp();
#pragma unroll
    for (int p = 0; p < RB; ++p)
#pragma unroll
      for (int o = LPR / 2; o > 0; o >>= 1) acc[p] += __shfl_xor_sync(kFull, acc[p], o);
    epi.post(row, live, acc, tl);
  }
}

// Where a phase reads and writes a level vector: this CTA's rows only (LOCAL, indexed from the
// CTA's first row), the whole vector replicated in every CTA of the cluster (REPLICA: a store
// goes to all CTAs' copies through distributed shared memory), or global memory (GLOBAL).
enum { VEC_LOCAL = 0, VEC_REPLICA = 1, VEC_GLOBAL = 2 };

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
  return r;
}
__device__ __forceinline__ void st_cluster(uint32_t addr, float v) {
  asm volatile("st.shared::cluster.f32 [%0], %1;\n" ::"r"(addr), "f"(v) : "memory");
}
__device__ __forceinline__ void st_cluster(uint32_t addr, double v) {
  asm volatile("st.shared::cluster.f64 [%0], %1;\n" ::"r"(addr), "d"(v) : "memory");
}
// Stores v at the same shared-memory offset in every CTA of the cluster (this one included).
template <typename V>
__device__ __forceinline__ void broadcast(V* local, V v) {
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(local);
  const uint32_t n = gridDim.x;
  for (uint32_t k = 0; k < n; ++k) {
    uint32_t remote;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(remote) : "r"(a), "r"(k));
    st_cluster(remote, v);
  }
}

template <typename V>
struct Vref {
  V* p;
  uint32_t row0;  // LOCAL: the CTA's first row
  int mode;
  __device__ __forceinline__ size_t at(uint32_t row, int q) const {
    return (size_t)(mode == VEC_LOCAL ? row - row0 : row) * 6 + q;
  }
  __device__ __forceinline__ V load(uint32_t row, int q) const {
    return mode == VEC_GLOBAL ? __ldcg(p + at(row, q)) : p[at(row, q)];
  }
  __device__ __forceinline__ void store(uint32_t row, int q, V v) const {
    if (mode == VEC_REPLICA)
      broadcast(p + at(row, q), v);
    else
      p[at(row, q)] = v;
  }
};

template <typename V>
__device__ __forceinline__ Vref<V> vref(V* p, uint32_t row0, int mode) {
  Vref<V> v;
  v.p = p;
  v.row0 = row0;
  v.mode = mode;
  return v;
}

// EpiAxpy through vector references.
template <typename V, int LPR, int OP>
struct TailAxpy {
  static constexpr int N = Parts<6, LPR>::N;
  Vref<V> y, b;
  V in[N];
  __device__ __forceinline__ void pre(uint32_t row, bool live, int tl) {
    if constexpr (OP != OP_SET) {
      if (!live) return;
#pragma unroll
      for (int k = 0; k < N; ++k) {
        int p = tl + k * LPR;
        if (p < 6) in[k] = OP == OP_RESIDUAL ? b.load(row, p) : y.load(row, p);
      }
    }
  }
  __device__ __forceinline__ void post(uint32_t row, bool live, const V (&acc)[6], int tl) {
    if (!live) return;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      int p = tl + k * LPR;
      if (p >= 6) continue;
      V sum = pick<V, 6>(acc, p);
      if (OP == OP_SET) y.store(row, p, sum);
      if (OP == OP_RESIDUAL) y.store(row, p, in[k] - sum);
      if (OP == OP_ADD) y.store(row, p, in[k] + sum);
    }
  }
};

// EpiCheb through vector references; D^-1 from the staged rows (first row `row0`). With
// `has_outer` the step stores outer_out = outer_in + (x + d_new) instead of x.
template <typename S, typename V, int LPR>
struct TailCheb {
  static constexpr int N = Parts<6, LPR>::N;
  const S* dinv;
  uint32_t row0;
  Vref<V> d_old, d_new, r, x, outer_in, outer_out;
  bool has_outer;
  V keep, step;
  V rv[6];
  V dv[N], xv[N], ov[N];
  S di[N][6];
  __device__ __forceinline__ void pre(uint32_t row, bool live, int tl) {
    if (!live) return;
    const size_t local = (size_t)(row - row0) * 36;
#pragma unroll
    for (int q = 0; q < 6; ++q) rv[q] = r.load(row, q);
#pragma unroll
    for (int k = 0; k < N; ++k) {
      int p = tl + k * LPR;
      if (p >= 6) continue;
#pragma unroll
      for (int q = 0; q < 6; ++q) di[k][q] = dinv[local + p * 6 + q];
      dv[k] = d_old.load(row, p);
      xv[k] = x.load(row, p);
      if (has_outer) ov[k] = outer_in.load(row, p);
    }
  }
  __device__ __forceinline__ void post(uint32_t row, bool live, const V (&acc)[6], int tl) {
    if (!live) return;
    V rn[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) rn[q] = rv[q] - acc[q];
#pragma unroll
    for (int k = 0; k < N; ++k) {
      int p = tl + k * LPR;
      if (p >= 6) continue;
      V z = V(0);
#pragma unroll
      for (int q = 0; q < 6; ++q) z += V(di[k][q]) * rn[q];
      V dn = keep * dv[k] + step * z;
      r.store(row, p, pick<V, 6>(rn, p));
      d_new.store(row, p, dn);
      V xn = xv[k] + dn;
      if (has_outer)
        outer_out.store(row, p, ov[k] + xn);
      else
        x.store(row, p, xn);
    }
  }
};

// This CTA's staged data and vectors: its rows of the level operator, prolongator and D^-1, its
// rows of the restriction and of the coarse inverse; replicas of the gathered vectors (d0, d1, x,
// res, and the coarse b and x); its own rows of r, post_x, tmp and b.
template <typename S, typename V>
struct TailLocal {
  LocalMat<S> a, p, r;
  const S* dinv;
  const double* inv;
  uint32_t c0, c1;  // coarse rows of the inverse
  V *d0, *d1, *x, *res, *cb, *cx;  // replicas
  V *r_own, *post_x, *tmp, *b;     // own rows
};

template <typename V, int OP, typename S>
__device__ __forceinline__ void tail_axpy(const LocalMat<S>& A, int lanes, const V* x, Vref<V> y, Vref<V> b) {
  switch (lanes) {
    case 4: { TailAxpy<V, 4, OP> e{y, b, {}}; tail_rows<S, V, 4>(A, x, e); break; }
    case 8: { TailAxpy<V, 8, OP> e{y, b, {}}; tail_rows<S, V, 8>(A, x, e); break; }
    case 16: { TailAxpy<V, 16, OP> e{y, b, {}}; tail_rows<S, V, 16>(A, x, e); break; }
    default: { TailAxpy<V, 32, OP> e{y, b, {}}; tail_rows<S, V, 32>(A, x, e); break; }
  }
}

template <typename S, typename V, int LPR>
__device__ __forceinline__ void tail_cheb_lpr(const TailLocal<S, V>& l, V* d_old, V* d_new, Vref<V> x, bool has_outer,
                                              Vref<V> outer_in, Vref<V> outer_out, V keep, V step) {
  TailCheb<S, V, LPR> e;
  e.dinv = l.dinv;
  e.row0 = l.a.row0;
  e.d_old = vref(d_old, 0, VEC_REPLICA);
  e.d_new = vref(d_new, 0, VEC_REPLICA);
  e.r = vref(l.r_own, l.a.row0, VEC_LOCAL);
  e.x = x;
  e.outer_in = outer_in;
  e.outer_out = outer_out;
  e.has_outer = has_outer;
  e.keep = keep;
  e.step = step;
  tail_rows<S, V, LPR>(l.a, d_old, e);
}

template <typename S, typename V>
__device__ __forceinline__ void tail_cheb(int lanes, const TailLocal<S, V>& l, V* d_old, V* d_new, Vref<V> x,
                                          bool has_outer, Vref<V> outer_in, Vref<V> outer_out, V keep, V step) {
  switch (lanes) {
    case 4: tail_cheb_lpr<S, V, 4>(l, d_old, d_new, x, has_outer, outer_in, outer_out, keep, step); break;
    case 8: tail_cheb_lpr<S, V, 8>(l, d_old, d_new, x, has_outer, outer_in, outer_out, keep, step); break;
    case 16: tail_cheb_lpr<S, V, 16>(l, d_old, d_new, x, has_outer, outer_in, outer_out, keep, step); break;
    default: tail_cheb_lpr<S, V, 32>(l, d_old, d_new, x, has_outer, outer_in, outer_out, keep, step); break;
  }
}

// The smoother of enqueue_smooth on level s: the start (cheb_start_kernel, term for term) on the
// CTA's rows of b into x, then the steps; with an outer vector the last step stores
// outer_out = outer_in + x. Every phase that stores into replicas ends at a cluster barrier, so
// no CTA leaves while another may still store into its shared memory.
template <typename S, typename V>
__device__ __forceinline__ void tail_smooth(const TailArgs<S, V>& t, const TailLocal<S, V>& l, const V* b_own,
                                            Vref<V> x, bool has_outer, Vref<V> outer_in, Vref<V> outer_out) {
  for (uint32_t lr = threadIdx.x; lr < l.a.rows; lr += blockDim.x) {
    const uint32_t row = l.a.row0 + lr;
    const S* di = l.dinv + (size_t)lr * 36;
    V bv[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      bv[q] = b_own[(size_t)lr * 6 + q];
      l.r_own[(size_t)lr * 6 + q] = bv[q];
    }
#pragma unroll
    for (int p = 0; p < 6; ++p) {
      V z = V(0);
#pragma unroll
      for (int q = 0; q < 6; ++q) z += V(di[p * 6 + q]) * bv[q];
      V dv = z / t.theta;
      broadcast(l.d0 + (size_t)row * 6 + p, dv);
      x.store(row, p, dv);
    }
  }
  cluster_barrier();
  for (uint32_t k = 0; k < t.nsteps; ++k) {
    const bool last = k + 1 == t.nsteps;
    V* d_old = (k & 1) ? l.d1 : l.d0;
    V* d_new = (k & 1) ? l.d0 : l.d1;
    tail_cheb<S, V>(t.a.lanes, l, d_old, d_new, x, last && has_outer, outer_in, outer_out, t.keep[k], t.step[k]);
    cluster_barrier();
  }
  if (has_outer && t.nsteps == 0) {
    for (uint32_t i = threadIdx.x; i < l.a.rows * 6; i += blockDim.x) {
      const uint32_t row = l.a.row0 + i / 6;
      const int q = (int)(i % 6);
      outer_out.store(row, q, outer_in.load(row, q) + x.load(row, q));
    }
    cluster_barrier();
  }
}

template <typename S, typename V>
__device__ __forceinline__ void tail_kernel(TailArgs<S, V> t) {
  if (*t.status != ST_ACTIVE) return;  // one word for the whole cluster: every CTA leaves or none
  // Lay out this CTA's shared memory (the layout tail_cta_bytes sizes on the host) and stage its
  // rows. The replicas come first, so a store into another CTA's replica lands at the same offset.
  extern __shared__ __align__(16) unsigned char tail_smem[];
  const uint32_t n = gridDim.x, i = cluster_rank();
  const uint32_t a0 = tail_share(t.a.rows, n, i), a1 = tail_share(t.a.rows, n, i + 1);
  const uint32_t r0 = tail_share(t.r.rows, n, i), r1 = tail_share(t.r.rows, n, i + 1);
  const uint32_t nv = t.a.rows * 6;
  TailLocal<S, V> l;
  l.c0 = tail_share(t.nc, n, i);
  l.c1 = tail_share(t.nc, n, i + 1);
  unsigned char* at = tail_smem;
  auto take = [&](size_t count) {
    V* p = reinterpret_cast<V*>(at);
    at += tail_align(count * sizeof(V));
    return p;
  };
  l.d0 = take(nv);
  l.d1 = take(nv);
  l.x = take(nv);
  l.res = take(nv);
  l.cb = take(t.nc);
  l.cx = take(t.nc);
  l.a = tail_stage(t.a, a0, a1, at);
  l.p = tail_stage(t.p, a0, a1, at);
  l.r = tail_stage(t.r, r0, r1, at);
  {
    S* d = reinterpret_cast<S*>(at);
    at += tail_align((size_t)(a1 - a0) * 36 * sizeof(S));
    stage16(reinterpret_cast<float4*>(d), reinterpret_cast<const float4*>(t.dinv + (size_t)a0 * 36),
            (size_t)(a1 - a0) * 36 * sizeof(S) / 16);
    l.dinv = d;
    double* v = reinterpret_cast<double*>(at);
    at += tail_align((size_t)(l.c1 - l.c0) * t.nc * 8);
    for (size_t k = threadIdx.x; k < (size_t)(l.c1 - l.c0) * t.nc; k += blockDim.x)
      v[k] = __ldg(t.inv + (size_t)l.c0 * t.nc + k);
    l.inv = v;
  }
  const size_t own = (size_t)(a1 - a0) * 6;
  l.r_own = take(own);
  l.post_x = take(own);
  l.tmp = take(own);
  l.b = take(own);
  for (size_t k = threadIdx.x; k < own; k += blockDim.x) l.b[k] = __ldcg(t.b + (size_t)a0 * 6 + k);
  __syncthreads();
  // Every CTA of the cluster is running and laid out before any store reaches another's replicas.
  cluster_barrier();

  const Vref<V> x_rep = vref(l.x, 0, VEC_REPLICA), none = vref((V*)nullptr, 0, VEC_LOCAL);
  tail_smooth<S, V>(t, l, l.b, x_rep, false, none, none);
  tail_axpy<V, OP_RESIDUAL>(l.a, t.a.lanes, l.x, vref(l.res, 0, VEC_REPLICA), vref(l.b, a0, VEC_LOCAL));
  cluster_barrier();
  tail_axpy<V, OP_SET>(l.r, t.r.lanes, l.res, vref(l.cb, 0, VEC_REPLICA), none);
  cluster_barrier();
  {
    // coarse_solve_kernel, term for term
    const uint32_t warps = blockDim.x >> 5;
    const int lane = threadIdx.x & 31;
    for (uint32_t lr = threadIdx.x >> 5; lr < l.c1 - l.c0; lr += warps) {
      const double* a = l.inv + (size_t)lr * t.nc;
      double s = 0.0;
      for (uint32_t j = lane; j < t.nc; j += 32) s += a[j] * (double)l.cb[j];
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
      if (lane == 0) broadcast(l.cx + l.c0 + lr, V(s));
    }
  }
  cluster_barrier();
  tail_axpy<V, OP_ADD>(l.p, t.p.lanes, l.cx, x_rep, none);
  cluster_barrier();
  tail_axpy<V, OP_RESIDUAL>(l.a, t.a.lanes, l.x, vref(l.tmp, a0, VEC_LOCAL), vref(l.b, a0, VEC_LOCAL));
  cluster_barrier();
  tail_smooth<S, V>(t, l, l.tmp, vref(l.post_x, a0, VEC_LOCAL), true, x_rep, vref(t.x, 0, VEC_GLOBAL));
}

// Shared memory CTA i of n needs (the layout of tail_kernel), from the host row starts of the
// level operator, prolongator and restriction.
inline size_t tail_cta_bytes(const std::vector<uint32_t>& a_starts, const std::vector<uint32_t>& p_starts,
                             const std::vector<uint32_t>& r_starts, uint32_t nc, uint32_t n, uint32_t i,
                             size_t value_bytes, size_t vector_bytes) {
  const uint32_t rows = (uint32_t)a_starts.size() - 1, crows = (uint32_t)r_starts.size() - 1;
  const uint32_t a0 = tail_share(rows, n, i), a1 = tail_share(rows, n, i + 1);
  const uint32_t r0 = tail_share(crows, n, i), r1 = tail_share(crows, n, i + 1);
  const uint32_t c0 = tail_share(nc, n, i), c1 = tail_share(nc, n, i + 1);
  const size_t nv = (size_t)rows * 6, own = (size_t)(a1 - a0) * 6;
  return 4 * tail_align(nv * vector_bytes) + 2 * tail_align((size_t)nc * vector_bytes) +
         tail_mat_bytes(a1 - a0, a_starts[a1] - a_starts[a0], value_bytes) +
         tail_mat_bytes(a1 - a0, p_starts[a1] - p_starts[a0], value_bytes) +
         tail_mat_bytes(r1 - r0, r_starts[r1] - r_starts[r0], value_bytes) +
         tail_align((size_t)(a1 - a0) * 36 * value_bytes) + tail_align((size_t)(c1 - c0) * nc * 8) +
         4 * tail_align(own * vector_bytes);
}

// ------------------------------------------------------------ smoother starts fused into products
// A level's smoother starts from zero on a right-hand side that a product has just made: the
// residual b - A x before the post-smoother, the restriction R r before a coarser level's
// pre-smoother. The start (cheb_start_kernel, term for term: r = b; d = (D^-1 b) / theta; x = d)
// is done in that product's epilogue, from the row's freshly summed values, so the start needs
// no launch of its own and the post-smoother's right-hand side never goes to memory.
template <typename S, typename V>
struct StartArgs {
  const S* dinv;
  V* b_out;  // the right-hand side, when the level reads it again (the restricted b); or null
  V* r;
  V* d;
  V* x;
  V theta;
};

// Component p of a block row's start from the row's right-hand side values bv.
template <typename S, typename V, int RB>
__device__ __forceinline__ void start_part(const StartArgs<S, V>& a, uint32_t row, int p, const V (&bv)[RB]) {
  const size_t base = (size_t)row * RB;
  if (a.b_out) a.b_out[base + p] = bv[p];
  a.r[base + p] = bv[p];
  V z = V(0);
#pragma unroll
  for (int q = 0; q < RB; ++q) z += V(a.dinv[base * RB + p * RB + q]) * bv[q];
  V dv = z / a.theta;
  a.d[base + p] = dv;
  a.x[base + p] = dv;
}

// SELL-32 (one thread per block row).
template <typename S, typename V, int RB, int OP>
struct SellStart {
  StartArgs<S, V> a;
  const V* __restrict__ b;
  V in[RB];
  __device__ __forceinline__ void pre(uint32_t row, bool live) {
    if (OP != OP_RESIDUAL || !live) return;
#pragma unroll
    for (int q = 0; q < RB; ++q) in[q] = b[(size_t)row * RB + q];
  }
  __device__ __forceinline__ void post(uint32_t row, bool live, uint32_t, const V (&acc)[RB], const V (&)[RB]) {
    if (!live) return;
    V bv[RB];
#pragma unroll
    for (int q = 0; q < RB; ++q) bv[q] = OP == OP_RESIDUAL ? in[q] - acc[q] : acc[q];
#pragma unroll
    for (int p = 0; p < RB; ++p) start_part<S, V, RB>(a, row, p, bv);
  }
};

template <typename S, typename V, int RB, int CB, int OP>
__device__ __forceinline__ void sell_start_kernel(SellOp<S> A, const V* __restrict__ x, const V* __restrict__ b,
                                                  StartArgs<S, V> a, const int* __restrict__ status) {
  SellStart<S, V, RB, OP> epi;
  epi.a = a;
  epi.b = b;
  sell_rows<S, V, RB, CB, false>(A, x, epi, StatusGate{status});
}

// Split rows (lane 6 m + p: scalar row p of block row m); the six values of a block row meet by
// shuffles, as in SplitCheb.
template <typename S, typename V, int OP>
struct SplitStart {
  StartArgs<S, V> a;
  const V* __restrict__ b;
  V in;
  __device__ __forceinline__ void pre(uint32_t row, uint32_t part, bool live) {
    if (OP == OP_RESIDUAL && live) in = b[(size_t)row * 6 + part];
  }
  __device__ __forceinline__ void post(uint32_t row, uint32_t part, bool live, V acc) {
    const V t = live ? (OP == OP_RESIDUAL ? in - acc : acc) : V(0);
    const uint32_t first = (threadIdx.x & 31) - part;
    V bv[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) bv[q] = __shfl_sync(kFull, t, (first + q) & 31);
    if (!live) return;
    start_part<S, V, 6>(a, row, (int)part, bv);
  }
};

template <typename S, typename V, int CB, int OP>
__device__ __forceinline__ void split_start_kernel(SellOp<S> A, const V* __restrict__ x, const V* __restrict__ b,
                                                   StartArgs<S, V> a, const int* __restrict__ status) {
  SplitStart<S, V, OP> epi;
  epi.a = a;
  epi.b = b;
  epi.in = V(0);
  split_rows<S, V, CB>(A, x, epi, StatusGate{status});
}

// Row groups (LPR lanes per row): after the butterfly every lane holds the whole row.
template <typename S, typename V, int RB, int LPR, int OP>
struct EpiStart {
  StartArgs<S, V> a;
  const V* __restrict__ b;
  V in[RB];
  __device__ __forceinline__ void pre(uint32_t row, bool live, int) {
    if (OP != OP_RESIDUAL || !live) return;
#pragma unroll
    for (int q = 0; q < RB; ++q) in[q] = b[(size_t)row * RB + q];
  }
  __device__ __forceinline__ void post(uint32_t row, bool live, const V (&acc)[RB], const V (&)[RB], int tl) {
    if (!live) return;
    V bv[RB];
#pragma unroll
    for (int q = 0; q < RB; ++q) bv[q] = OP == OP_RESIDUAL ? in[q] - acc[q] : acc[q];
#pragma unroll
    for (int k = 0; k < Parts<RB, LPR>::N; ++k) {
      const int p = tl + k * LPR;
      if (p < RB) start_part<S, V, RB>(a, row, p, bv);
    }
  }
};

template <typename S, typename V, int RB, int CB, int LPR, int OP>
__device__ __forceinline__ void bsr_start_kernel(Op<S> A, const V* __restrict__ x, const V* __restrict__ b,
                                                 StartArgs<S, V> a, const int* __restrict__ status) {
  extern __shared__ __align__(16) char smem[];
  char* wbase = smem + (threadIdx.x >> 5) * 2 * slot_bytes(A);
  EpiStart<S, V, RB, LPR, OP> epi;
  epi.a = a;
  epi.b = b;
  run_groups<S, V, RB, CB, LPR, false>(A, x, wbase, epi, StatusGate{status});
}

struct SellDot {
  const double* __restrict__ p;
  double* __restrict__ ap;
  double local;
  double pv[3];
  __device__ __forceinline__ void pre(uint32_t row, bool live) {
    if (!live) return;
#pragma unroll
    for (int q = 0; q < 3; ++q) pv[q] = p[(size_t)row * 3 + q];
  }
  __device__ __forceinline__ void post(uint32_t row, bool live, uint32_t, const double (&acc)[3], const double (&)[3]) {
    if (!live) return;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      ap[(size_t)row * 3 + q] = acc[q];
      local += pv[q] * acc[q];
    }
  }
};

__device__ __forceinline__ void sell_pcg_spmv_dot_kernel(SellOp<double> A, const double* __restrict__ p,
                                                                      double* __restrict__ ap, double* partials,
                                                                      PcgState* st) {
  SellDot epi;
  epi.p = p;
  epi.ap = ap;
  epi.local = 0.0;
  if (!sell_rows<double, double, 3, 3, false>(A, p, epi, StatusGate{&st->status})) return;
  double v[1] = {epi.local}, total[1];
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

struct SellCheck {
  const double* __restrict__ b;
  double* __restrict__ r;
  double res2, bound2;
  double bv[3];
  __device__ __forceinline__ void pre(uint32_t row, bool live) {
    if (!live) return;
#pragma unroll
    for (int q = 0; q < 3; ++q) bv[q] = b[(size_t)row * 3 + q];
  }
  __device__ __forceinline__ void post(uint32_t row, bool live, uint32_t n, const double (&acc)[3], const double (&mag)[3]) {
    if (!live) return;
    const double eps = 2.220446049250313e-16;
    double terms = (double)(n * 3);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      double res = bv[q] - acc[q];
      r[(size_t)row * 3 + q] = res;
      res2 += res * res;
      double bound = terms * eps * mag[q];
      bound2 += bound * bound;
    }
  }
};

__device__ __forceinline__ void sell_pcg_check_kernel(SellOp<double> A, const double* __restrict__ x,
                                                                   const double* __restrict__ b, double* __restrict__ r,
                                                                   double* partials, PcgState* st) {
  SellCheck epi;
  epi.b = b;
  epi.r = r;
  epi.res2 = 0.0;
  epi.bound2 = 0.0;
  if (!sell_rows<double, double, 3, 3, true>(A, x, epi, CheckGate{st})) return;
  double v[2] = {epi.res2, epi.bound2}, total[2];
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

// ap = A p with the curvature p.ap.
template <int LPR>
struct EpiDot {
  static constexpr int N = Parts<3, LPR>::N;
  const double* __restrict__ p;
  double* __restrict__ ap;
  double local;
  double pv[N];
  __device__ __forceinline__ void pre(uint32_t row, bool live, int tl) {
    if (!live) return;
#pragma unroll
    for (int k = 0; k < N; ++k)
      if (tl + k * LPR < 3) pv[k] = p[(size_t)row * 3 + tl + k * LPR];
  }
  __device__ __forceinline__ void post(uint32_t row, bool live, const double (&acc)[3], const double (&)[3], int tl) {
    if (!live) return;
#pragma unroll
    for (int k = 0; k < N; ++k) {
      int q = tl + k * LPR;
      if (q >= 3) continue;
      double sum = pick<double, 3>(acc, q);
      ap[(size_t)row * 3 + q] = sum;
      local += pv[k] * sum;
    }
  }
};

// ap = A p on the f64 system with the curvature p.ap; then alpha = rz / curvature
// (pcg.rs:217-228).
template <int LPR>
__device__ __forceinline__ void pcg_spmv_dot_kernel(Op<double> A, const double* __restrict__ p,
                                                                 double* __restrict__ ap, double* partials, PcgState* st) {
  extern __shared__ __align__(16) char smem[];
  char* wbase = smem + (threadIdx.x >> 5) * 2 * slot_bytes(A);
  EpiDot<LPR> epi;
  epi.p = p;
  epi.ap = ap;
  epi.local = 0.0;
  if (!run_groups<double, double, 3, 3, LPR, false>(A, p, wbase, epi, StatusGate{&st->status})) return;
  double v[1] = {epi.local}, total[1];
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
__device__ __forceinline__ void pcg_update_kernel(uint32_t n, const double* __restrict__ p,
                                                               const double* __restrict__ ap, double* __restrict__ x,
                                                               double* __restrict__ r, double* partials, PcgState* st) {
  if (st->status != ST_ACTIVE) return;
  double alpha = st->alpha, na = -alpha;
  double local = 0.0;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i0 < n; i0 += kStrides * stride) {
    double pv[kStrides], av[kStrides], xv[kStrides], rv[kStrides];
#pragma unroll
    for (int k = 0; k < kStrides; ++k) {
      const size_t i = i0 + k * stride;
      const bool in = i < n;
      pv[k] = in ? p[i] : 0.0;
      av[k] = in ? ap[i] : 0.0;
      xv[k] = in ? x[i] : 0.0;
      rv[k] = in ? r[i] : 0.0;
    }
#pragma unroll
    for (int k = 0; k < kStrides; ++k) {
      const size_t i = i0 + k * stride;
      if (i >= n) break;
      x[i] = xv[k] + alpha * pv[k];
      double rn = rv[k] + na * av[k];
      r[i] = rn;
      local += rn * rn;
    }
  }
  double v[1] = {local}, total[1];
  if (finish_partials<1>(v, partials, &st->tickets[1], total) && threadIdx.x == 0) {
    st->iterations += 1;
    double rel = sqrt(total[0]) / st->rhs_norm;
    st->rel = rel;
    st->mode = rel <= st->tolerance ? MODE_CHECK : MODE_NORMAL;
  }
}

// r = b - A x with the rounding-floor row bounds (csr.rs:142-154).
template <int LPR>
struct EpiCheck {
  static constexpr int N = Parts<3, LPR>::N;
  const double* __restrict__ b;
  double* __restrict__ r;
  const uint32_t* __restrict__ starts;
  double res2, bound2;
  double bv[N];
  __device__ __forceinline__ void pre(uint32_t row, bool live, int tl) {
    if (!live) return;
#pragma unroll
    for (int k = 0; k < N; ++k)
      if (tl + k * LPR < 3) bv[k] = b[(size_t)row * 3 + tl + k * LPR];
  }
  __device__ __forceinline__ void post(uint32_t row, bool live, const double (&acc)[3], const double (&mag)[3], int tl) {
    if (!live) return;
    const double eps = 2.220446049250313e-16;
    double terms = (double)((starts[row + 1] - starts[row]) * 3);
#pragma unroll
    for (int k = 0; k < N; ++k) {
      int q = tl + k * LPR;
      if (q >= 3) continue;
      size_t i = (size_t)row * 3 + q;
      double res = bv[k] - pick<double, 3>(acc, q);
      r[i] = res;
      res2 += res * res;
      double bound = terms * eps * pick<double, 3>(mag, q);
      bound2 += bound * bound;
    }
  }
};

// The true residual when the recursive one reports convergence, with the rounding floor of the
// product (pcg.rs:234-255): r = b - A x; converge, or restart from it.
template <int LPR>
__device__ __forceinline__ void pcg_check_kernel(Op<double> A, const double* __restrict__ x,
                                                              const double* __restrict__ b, double* __restrict__ r,
                                                              double* partials, PcgState* st) {
  extern __shared__ __align__(16) char smem[];
  char* wbase = smem + (threadIdx.x >> 5) * 2 * slot_bytes(A);
  EpiCheck<LPR> epi;
  epi.b = b;
  epi.r = r;
  epi.starts = A.starts;
  epi.res2 = 0.0;
  epi.bound2 = 0.0;
  if (!run_groups<double, double, 3, 3, LPR, true>(A, x, wbase, epi, CheckGate{st})) return;
  double v[2] = {epi.res2, epi.bound2}, total[2];
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
__device__ __forceinline__ void pcg_dot_rz_kernel(uint32_t n, const double* __restrict__ r,
                                                               const Z* __restrict__ z, const double* __restrict__ ap,
                                                               double* partials, PcgState* st) {
  if (st->status != ST_ACTIVE) return;
  bool flex = st->flexible && st->mode == MODE_NORMAL;
  double rz = 0.0, apz = 0.0;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i0 < n; i0 += kStrides * stride) {
    double zv[kStrides], rv[kStrides], av[kStrides];
#pragma unroll
    for (int k = 0; k < kStrides; ++k) {
      const size_t i = i0 + k * stride;
      const bool in = i < n;
      zv[k] = in ? (double)z[i] : 0.0;
      rv[k] = in ? r[i] : 0.0;
      av[k] = in && flex ? ap[i] : 0.0;
    }
#pragma unroll
    for (int k = 0; k < kStrides; ++k) {
      if (i0 + k * stride >= n) break;
      rz += rv[k] * zv[k];
      if (flex) apz += av[k] * zv[k];
    }
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
__device__ __forceinline__ void pcg_update_p_kernel(uint32_t n, const Z* __restrict__ z, double* __restrict__ p, PcgState* st) {
  if (st->status != ST_ACTIVE) return;
  bool restart = st->mode == MODE_RESTART;
  double beta = st->beta;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i0 < n; i0 += kStrides * stride) {
    double zv[kStrides], pv[kStrides];
#pragma unroll
    for (int k = 0; k < kStrides; ++k) {
      const size_t i = i0 + k * stride;
      const bool in = i < n;
      zv[k] = in ? (double)z[i] : 0.0;
      pv[k] = in && !restart ? p[i] : 0.0;
    }
#pragma unroll
    for (int k = 0; k < kStrides; ++k) {
      const size_t i = i0 + k * stride;
      if (i >= n) break;
      p[i] = restart ? zv[k] : zv[k] + beta * pv[k];
    }
  }
}

// Initial state (Pcg::new, pcg.rs:135-164): x = 0, r = b, rhs norm; then reset_direction.
__device__ __forceinline__ void pcg_init_kernel(uint32_t n, const double* __restrict__ b, double* __restrict__ x,
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
__device__ __forceinline__ void jacobi_kernel(uint32_t n, const double* __restrict__ inv, const double* __restrict__ r,
                              double* __restrict__ z, const int* __restrict__ status) {
  if (*status != ST_ACTIVE) return;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) z[i] = r[i] * inv[i];
}

// ------------------------------------------------------------ launch helpers
int g_sm_count = 0;

int sm_count() {
  if (g_sm_count == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (g_sm_count <= 0) g_sm_count = 148;
  }
  return g_sm_count;
}

int grid_for_elems(size_t n) {
  size_t blocks = (n + kThreads - 1) / kThreads;
  size_t cap = (size_t)sm_count() * 8;
  return (int)std::max<size_t>(1, std::min(blocks, cap));
}

int grid_for_rows(size_t rows) {
  size_t blocks = (rows + kWarps - 1) / kWarps;
  return (int)std::max<size_t>(1, std::min(blocks, (size_t)sm_count() * 8));
}

// Launch shape of a grouped product: warps per block so a block stages at most about 72 KB, and
// a grid of whole waves (resident blocks per SM times SMs), never more warps than groups.
struct Shape {
  int threads, grid;
  size_t smem;
};

template <typename S>
Shape shape_of(const Op<S>& A, bool reduction) {
  size_t per_warp = 2 * (size_t)slot_bytes(A);
  int warps = (int)std::max<size_t>(1, std::min<size_t>(kWarps, kSmemPerBlockTarget / per_warp));
  size_t smem = per_warp * warps;
  // 228 KB of shared memory per SM, 1 KB of it reserved per resident block.
  int per_sm = (int)std::max<size_t>(1, std::min<size_t>(2048 / (32 * warps), (228 * 1024) / (smem + 1024)));
  size_t want = (A.ngroups + warps - 1) / warps;
  size_t grid = std::min<size_t>(want, (size_t)sm_count() * per_sm);
  if (reduction) grid = std::min<size_t>((size_t)sm_count() * per_sm, (size_t)kReduceBlocks * 2);
  return {32 * warps, (int)std::max<size_t>(1, grid), smem};
}


template <typename S, typename V, int RB, int CB, int LPR, int OP>
void launch_bsr_lpr(const DevBsr& m, const V* x, V* y, const V* b, const int* status, cudaStream_t st) {
  Op<S> A = op_of<S>(m);
  Shape sh = shape_of(A, false);
  launch_body<bsr_kernel<S, V, RB, CB, LPR, OP>>(sh.grid, sh.threads, sh.smem, st, A, x, y, b, status);
}

// The SELL-32 and split-row products run in blocks of two warps. The resident warps per SM do not
// change (at ~110 registers each scheduler's quarter of the register file holds four warps), but
// finer blocks even out the end of the grid: the SMs that finish early take the last slices two
// warps at a time (the finest Chebyshev step 41.7 -> 40.8 us), and level 1's ~2,000 slices spread
// evenly instead of two eight-warp blocks on some SMs and one on others (mixed solve 182.5 ->
// 181.7 ms). Same bits; FP64 unchanged.
constexpr int kSellThreads = 64;
inline int sell_threads() { return kSellThreads; }
inline int sell_grid(uint32_t nslices) {
  const int w = kSellThreads / 32;
  return (int)std::max<size_t>(1, (nslices + w - 1) / w);
}

int grid_for_slices(uint32_t nslices) {
  size_t blocks = (nslices + kWarps - 1) / kWarps;
  return (int)std::max<size_t>(1, std::min<size_t>(blocks, (size_t)sm_count() * 8));
}

template <typename S, typename V, int RB, int CB, int OP>
void launch_sell(const DevBsr& m, const V* x, V* y, const V* b, const int* status, cudaStream_t st) {
  launch_body<sell_kernel<S, V, RB, CB, OP>>(sell_grid(m.nslices), sell_threads(), 0, st, sell_of<S>(m), x, y, b, status);
}

template <typename S, typename V, int RB, int CB, int OP>
void launch_bsr(const DevBsr& m, const V* x, V* y, const V* b, const int* status, cudaStream_t st) {
  if (m.sell) {
    launch_sell<S, V, RB, CB, OP>(m, x, y, b, status, st);
    return;
  }
  switch (m.lanes_per_row) {
    case 4: launch_bsr_lpr<S, V, RB, CB, 4, OP>(m, x, y, b, status, st); break;
    case 8: launch_bsr_lpr<S, V, RB, CB, 8, OP>(m, x, y, b, status, st); break;
    case 16: launch_bsr_lpr<S, V, RB, CB, 16, OP>(m, x, y, b, status, st); break;
    default: launch_bsr_lpr<S, V, RB, CB, 32, OP>(m, x, y, b, status, st); break;
  }
}

template <typename S, typename V, int OP>
void launch_split(const DevBsr& m, const V* x, V* y, const V* b, const int* status, cudaStream_t st) {
  if (m.cb == 3)
    launch_body<split_kernel<S, V, 3, OP>>(sell_grid(m.nslices), sell_threads(), 0, st, sell_of<S>(m), x, y, b, status);
  else
    launch_body<split_kernel<S, V, 6, OP>>(sell_grid(m.nslices), sell_threads(), 0, st, sell_of<S>(m), x, y, b, status);
}

template <typename S, typename V, int RB, int OP>
void bsr_dispatch_cb(const DevBsr& m, const V* x, V* y, const V* b, const int* status, cudaStream_t st) {
  if (RB == 6 && m.split) {
    launch_split<S, V, OP>(m, x, y, b, status, st);
    return;
  }
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

template <typename S, typename V, int RB, int LPR>
void launch_cheb_step_lpr(const DevLevel& L, const V* d_old, V* d_new, V* r, V* x, V* outer, double keep, double step,
                          const int* status, cudaStream_t st) {
  Op<S> A = op_of<S>(L.a);
  Shape sh = shape_of(A, false);
  launch_body<cheb_step_kernel<S, V, RB, LPR>>(sh.grid, sh.threads, sh.smem, st, A, (const S*)L.dinv, d_old, d_new, r,
                                                x, outer, (V)keep, (V)step, status);
}

template <typename S, typename V, int RB>
void launch_cheb_step(const DevLevel& L, const V* d_old, V* d_new, V* r, V* x, V* outer, double keep, double step,
                      const int* status, cudaStream_t st) {
  if constexpr (RB == 6) {
    if (L.a.split) {
      launch_body<split_cheb_kernel<S, V>>(sell_grid(L.a.nslices), sell_threads(), 0, st, sell_of<S>(L.a),
                                           (const S*)L.dinv, d_old, d_new, r, x, outer, (V)keep, (V)step, status);
      return;
    }
  }
  if (L.a.sell) {
    launch_body<sell_cheb_kernel<S, V, RB>>(sell_grid(L.a.nslices), sell_threads(), 0, st,
        sell_of<S>(L.a), (const S*)L.dinv, d_old, d_new, r, x, outer, (V)keep, (V)step, status);
    return;
  }
  switch (L.a.lanes_per_row) {
    case 4: launch_cheb_step_lpr<S, V, RB, 4>(L, d_old, d_new, r, x, outer, keep, step, status, st); break;
    case 8: launch_cheb_step_lpr<S, V, RB, 8>(L, d_old, d_new, r, x, outer, keep, step, status, st); break;
    case 16: launch_cheb_step_lpr<S, V, RB, 16>(L, d_old, d_new, r, x, outer, keep, step, status, st); break;
    default: launch_cheb_step_lpr<S, V, RB, 32>(L, d_old, d_new, r, x, outer, keep, step, status, st); break;
  }
}

template <typename S, typename V, typename B, int RB>
void launch_cheb_start(const DevLevel& L, const B* b_in, V* b_out, V* r, V* d, V* x, double theta, const int* status,
                       cudaStream_t st) {
  launch_body<cheb_start_kernel<S, V, B, RB>>(grid_for_elems(L.a.rows), kThreads, 0, st,
      L.a.rows, (const S*)L.dinv, b_in, b_out, r, d, x, (V)theta, status);
}

// The product of `m` (a residual b - m x or a restriction m x) with the smoother start of the
// level that reads its result fused in (sell_start_kernel / split_start_kernel / bsr_start_kernel).
template <typename S, typename V, int RB, int CB, int OP>
void launch_start_rb(const DevBsr& m, const V* x, const V* b, const StartArgs<S, V>& a, const int* status,
                     cudaStream_t st) {
  if constexpr (RB == 6) {
    if (m.split) {
      launch_body<split_start_kernel<S, V, CB, OP>>(sell_grid(m.nslices), sell_threads(), 0, st, sell_of<S>(m), x, b,
                                                    a, status);
      return;
    }
  }
  if (m.sell) {
    launch_body<sell_start_kernel<S, V, RB, CB, OP>>(sell_grid(m.nslices), sell_threads(), 0, st, sell_of<S>(m), x, b,
                                                     a, status);
    return;
  }
  Op<S> A = op_of<S>(m);
  Shape sh = shape_of(A, false);
  switch (m.lanes_per_row) {
    case 4: launch_body<bsr_start_kernel<S, V, RB, CB, 4, OP>>(sh.grid, sh.threads, sh.smem, st, A, x, b, a, status); break;
    case 8: launch_body<bsr_start_kernel<S, V, RB, CB, 8, OP>>(sh.grid, sh.threads, sh.smem, st, A, x, b, a, status); break;
    case 16: launch_body<bsr_start_kernel<S, V, RB, CB, 16, OP>>(sh.grid, sh.threads, sh.smem, st, A, x, b, a, status); break;
    default: launch_body<bsr_start_kernel<S, V, RB, CB, 32, OP>>(sh.grid, sh.threads, sh.smem, st, A, x, b, a, status); break;
  }
}

template <typename S, typename V, int OP>
void launch_start_product(const DevBsr& m, const V* x, const V* b, const StartArgs<S, V>& a, const int* status,
                          cudaStream_t st) {
  if (m.rb == 3)
    launch_start_rb<S, V, 3, 3, OP>(m, x, b, a, status, st);
  else if (m.cb == 3)
    launch_start_rb<S, V, 6, 3, OP>(m, x, b, a, status, st);
  else
    launch_start_rb<S, V, 6, 6, OP>(m, x, b, a, status, st);
}

template <typename S, typename V>
StartArgs<S, V> start_args(const DevLevel& L, V* b_out, V* x) {
  StartArgs<S, V> a;
  a.dinv = (const S*)L.dinv;
  a.b_out = b_out;
  a.r = (V*)L.res;
  a.d = (V*)L.d0;
  a.x = x;
  a.theta = (V)L.theta;
  return a;
}

// The smoother from a zero guess on right-hand side b into x (cycle.rs:570-651). `outer`, when
// given, receives x += (smoothed x) at the last step instead of storing x.
template <typename S, typename V, typename B>
void enqueue_smooth(DeviceSolver& s, DevLevel& L, const B* b_in, V* b_out, V* x, V* outer, const int* status,
                    bool started = false) {
  cudaStream_t st = s.stream;
  V* r = (V*)L.res;
  V* d[2] = {(V*)L.d0, (V*)L.d1};
  if (!started) {  // else the product that made b_in did the start
    if (L.a.rb == 3)
      launch_cheb_start<S, V, B, 3>(L, b_in, b_out, r, d[0], x, L.theta, status, st);
    else
      launch_cheb_start<S, V, B, 6>(L, b_in, b_out, r, d[0], x, L.theta, status, st);
    s.launches_per_iteration++;
  }
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
    launch_body<add_kernel<V>>(grid_for_elems(L.n), kThreads, 0, st, L.n, outer, x, status);
    s.launches_per_iteration++;
  }
}

template <typename S>
TailMat<S> tail_mat(const DevBsr& m) {
  TailMat<S> t;
  t.starts = m.starts;
  t.cols = m.cols;
  t.vals = (const S*)m.vals;
  t.rows = m.rows;
  t.lanes = m.lanes_per_row;
  return t;
}

// Levels li and li + 1 (the coarsest, factored) as one cluster launch of tail_kernel.
template <typename S, typename V>
void enqueue_tail(DeviceSolver& s, size_t li, const int* status) {
  DevLevel& L = s.levels[li];
  DevLevel& C = s.levels[li + 1];
  TailArgs<S, V> t = {};
  t.a = tail_mat<S>(L.a);
  t.r = tail_mat<S>(L.r);
  t.p = tail_mat<S>(L.p);
  t.dinv = (const S*)L.dinv;
  t.inv = C.coarse_inverse;
  t.nc = C.n;
  t.nsteps = (uint32_t)L.steps.size();
  t.theta = (V)L.theta;
  for (size_t k = 0; k < L.steps.size(); ++k) {
    t.keep[k] = (V)L.steps[k].first;
    t.step[k] = (V)L.steps[k].second;
  }
  t.b = (const V*)L.b;
  t.x = (V*)L.x;
  t.status = status;
  launch_body_cluster<tail_kernel<S, V>, tail_threads<V>()>(dim3(s.tail_cluster), s.tail_smem, s.stream, t);
  s.launches_per_iteration++;
}

// CTAs of the tail's cluster on this device and their shared memory: 16 (a non-portable size)
// when each CTA's share fits kTailMaxSmem and the device can place such a cluster, else 8, else
// 0 (no tail). `hs` is the fused level, `hc` the coarsest.
template <typename S, typename V>
unsigned tail_cluster_size(const HostLevel& hs, const HostLevel& hc, size_t* smem) {
  typedef BodyTraits<decltype(&tail_kernel<S, V>)> T;
  const void* single = T::template single_n<tail_kernel<S, V>, tail_threads<V>()>();
  const void* batched = T::template batched_n<tail_kernel<S, V>, tail_threads<V>()>();
  // restriction row starts: the prolongator's blocks counted per coarse row
  std::vector<uint32_t> r_starts(hc.a.rows + 1, 0);
  for (uint32_t c : hs.p.cols) r_starts[c + 1] += 1;
  for (size_t i = 0; i < hc.a.rows; ++i) r_starts[i + 1] += r_starts[i];
  const uint32_t nc = (uint32_t)(hc.a.rows * hc.a.rb);
  cudaFuncSetAttribute(single, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  cudaFuncSetAttribute(batched, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  for (unsigned c : {16u, 8u}) {
    size_t bytes = 0;
    for (unsigned i = 0; i < c; ++i)
      bytes = std::max(bytes, tail_cta_bytes(hs.a.starts, hs.p.starts, r_starts, nc, c, i, sizeof(S), sizeof(V)));
    if (bytes > kTailMaxSmem) continue;
    cudaFuncSetAttribute(single, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    cudaFuncSetAttribute(batched, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = c;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c);
    cfg.blockDim = dim3(tail_threads<V>());
    cfg.dynamicSmemBytes = bytes;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, single, &cfg) == cudaSuccess && clusters > 0) {
      *smem = bytes;
      return c;
    }
    cudaGetLastError();
  }
  return 0;
}

// One V-cycle from level `li` (cycle.rs:461-539). B is the type of the right-hand side; an f64
// right-hand side reaching an f32 level is rounded into b_store first.
template <typename S, typename V, typename B>
void enqueue_cycle(DeviceSolver& s, size_t li, const B* rhs, V* b_store, V* x, const int* status,
                   bool started = false) {
  if ((int)li == s.tail_level) {
    enqueue_tail<S, V>(s, li, status);
    return;
  }
  DevLevel& L = s.levels[li];
  cudaStream_t st = s.stream;
  if (!L.has_p) {
    if (L.has_factor) {
      const V* bv = (const V*)rhs;
      if (b_store) {
        launch_body<convert_kernel<B, V>>(grid_for_elems(L.n), kThreads, 0, st, L.n, rhs, b_store, status);
        s.launches_per_iteration++;
        bv = b_store;
      }
      launch_body<coarse_solve_kernel<V>>(grid_for_rows(L.n), kThreads, 0, st, L.n, L.coarse_inverse, bv, x, status);
      s.launches_per_iteration++;
    } else {
      enqueue_smooth<S, V, B>(s, L, rhs, b_store, x, nullptr, status, started);
    }
    return;
  }
  enqueue_smooth<S, V, B>(s, L, rhs, b_store, x, nullptr, status, started);
  const V* b = b_store ? (const V*)b_store : (const V*)rhs;
  DevLevel& C = s.levels[li + 1];
  bsr_dispatch<S, V, OP_RESIDUAL>(L.a, x, (V*)L.res, b, status, st);
  // The restriction; when the coarser level starts with its smoother, that start is fused in.
  const bool fuse = (int)(li + 1) != s.tail_level && (C.has_p || !C.has_factor);
  if (fuse)
    launch_start_product<S, V, OP_SET>(L.r, (const V*)L.res, (const V*)nullptr,
                                       start_args<S, V>(C, (V*)C.b, (V*)C.x), status, st);
  else
    bsr_dispatch<S, V, OP_SET>(L.r, (const V*)L.res, (V*)C.b, nullptr, status, st);
  s.launches_per_iteration += 2;
  enqueue_cycle<S, V, V>(s, li + 1, (const V*)C.b, nullptr, (V*)C.x, status, fuse);
  bsr_dispatch<S, V, OP_ADD>(L.p, (const V*)C.x, x, nullptr, status, st);
  // The residual b - A x with the post-smoother's start fused in (its right-hand side stays in
  // registers).
  launch_start_product<S, V, OP_RESIDUAL>(L.a, (const V*)x, b, start_args<S, V>(L, (V*)nullptr, (V*)L.post_x),
                                          status, st);
  s.launches_per_iteration += 2;
  enqueue_smooth<S, V, V>(s, L, (const V*)nullptr, nullptr, (V*)L.post_x, x, status, true);
}

// z = M r for the solver's r (f64) into z (f64) or z32.
void enqueue_precondition(DeviceSolver& s, const double* r, double* z, float* z32, const int* status) {
  if (!s.multigrid) {
    launch_body<jacobi_kernel>(grid_for_elems(s.n), kThreads, 0, s.stream, s.n, s.jacobi, r, z, status);
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

template <int LPR>
void launch_pcg_spmv_lpr(DeviceSolver& s) {
  Op<double> A = op_of<double>(s.system);
  Shape sh = shape_of(A, true);
  launch_body<pcg_spmv_dot_kernel<LPR>>(sh.grid, sh.threads, sh.smem, s.stream, A, s.p, s.ap, s.partials, s.state);
  launch_body<pcg_update_kernel>(kReduceBlocks, kReduceThreads, 0, s.stream, s.n, s.p, s.ap, s.x, s.r, s.partials, s.state);
  launch_body<pcg_check_kernel<LPR>>(sh.grid, sh.threads, sh.smem, s.stream, A, s.x, s.rhs, s.r, s.partials, s.state);
}

}  // namespace

sf_status cuda_check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return SF_OK;
  char msg[200];
  std::snprintf(msg, sizeof(msg), "%s: %s", what, cudaGetErrorString(e));
  if (e == cudaErrorMemoryAllocation) return fail(SF_DEVICE_MEMORY_BUDGET, msg);
  return fail(SF_CUDA_ERROR, msg);
}

// Pinned host memory is never returned: freeing it synchronizes the whole device. Per host thread
// a grow-only scratch buffer (earlier, smaller buffers stay allocated and valid), and a shared
// pool of fixed 512-byte slots for per-study state read-backs.
namespace {
std::mutex g_slot_mutex;
std::vector<void*> g_free_slots;
std::mutex g_pool_mutex;
std::vector<std::pair<void*, size_t>> g_pool_free;    // returned buffers
std::vector<std::pair<void*, size_t>> g_pool_sizes;   // every buffer made
}  // namespace

void* pinned_acquire(size_t bytes) {
  bytes = std::max<size_t>(bytes, 1);
  std::lock_guard<std::mutex> lock(g_pool_mutex);
  size_t best = SIZE_MAX;
  for (size_t i = 0; i < g_pool_free.size(); ++i)
    if (g_pool_free[i].second >= bytes && (best == SIZE_MAX || g_pool_free[i].second < g_pool_free[best].second))
      best = i;
  if (best != SIZE_MAX) {
    void* p = g_pool_free[best].first;
    g_pool_free[best] = g_pool_free.back();
    g_pool_free.pop_back();
    return p;
  }
  const size_t want = (bytes + ((size_t)1 << 20) - 1) & ~(((size_t)1 << 20) - 1);  // whole MiB
  void* p = nullptr;
  if (cudaMallocHost(&p, want) != cudaSuccess) return nullptr;
  g_pool_sizes.push_back({p, want});
  return p;
}

void pinned_return(void* buffer) {
  if (!buffer) return;
  std::lock_guard<std::mutex> lock(g_pool_mutex);
  for (auto& b : g_pool_sizes)
    if (b.first == buffer) {
      g_pool_free.push_back(b);
      return;
    }
}

void* pinned_slot() {
  std::lock_guard<std::mutex> lock(g_slot_mutex);
  if (g_free_slots.empty()) {
    const size_t n = 128;
    void* p = nullptr;
    if (cudaMallocHost(&p, n * kPinnedSlotBytes) != cudaSuccess) return nullptr;
    for (size_t i = 0; i < n; ++i) g_free_slots.push_back((char*)p + i * kPinnedSlotBytes);
  }
  void* s = g_free_slots.back();
  g_free_slots.pop_back();
  return s;
}

void pinned_release(void* slot) {
  if (!slot) return;
  std::lock_guard<std::mutex> lock(g_slot_mutex);
  g_free_slots.push_back(slot);
}

// Device memory comes from the device's stream-ordered pool: an allocation or a free is ordered on
// the solver's stream and never waits for the rest of the device (cudaFree would synchronize the
// whole device, stalling every other study in flight). The pool keeps freed memory for reuse
// instead of returning it at each synchronization.
void pool_setup(int device) {
  static std::mutex mu;
  static bool done[64] = {};
  std::lock_guard<std::mutex> lock(mu);
  if (device < 0 || device >= 64 || done[device]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    // Reserve a first slab now (an eighth of the free memory, at most 8 GiB), once: growing the
    // pool later maps new memory inside a study's build, and such a call was measured blocking
    // the host for up to 0.8 s.
    size_t free_bytes = 0, total = 0;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    if (cudaMemGetInfo(&free_bytes, &total) == cudaSuccess) {
      const size_t slab = std::min<size_t>(free_bytes / 8, (size_t)8 << 30);
      cudaStream_t st = nullptr;
      void* p = nullptr;
      if (slab && cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess) {
        if (cudaMallocAsync(&p, slab, st) == cudaSuccess) cudaFreeAsync(p, st);
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
      }
      cudaGetLastError();
    }
    cudaSetDevice(prev);
  }
  done[device] = true;
}

sf_status dev_alloc(DeviceSolver& s, void** ptr, size_t bytes) {
  // 64 bytes of slack: the staged loads read whole 16-byte chunks past an array's last value.
  size_t padded = bytes + 64;
  pool_setup(s.device);
  cudaError_t e = cudaMallocAsync(ptr, padded, s.stream);
  if (e != cudaSuccess) return cuda_check(e, "cudaMallocAsync");
  cudaMemsetAsync(*ptr, 0, padded, s.stream);
  s.owned.push_back({*ptr, padded});
  s.bytes += padded;
  return SF_OK;
}

bool wants_sell(const DevBsr& m, uint64_t sell_min_rows) {
  // A warp stages two row groups at once; a group is at least one row, so an operator with rows
  // too long to stage (the transposes of wide prolongators) runs one thread per row instead.
  const size_t slot = ((m.group_bytes + 31) & ~15u) + ((m.group_blocks * 4 + 31) & ~15u) +
                      (((m.group_rows + 1) * 4 + 31) & ~15u);
  return m.rows >= sell_min_rows || 2 * slot > kMaxStagePerWarp;
}

bool wants_split(const DevBsr& m, bool uniform_lanes) {
  return !uniform_lanes && m.rb == 6 && (m.cb == 3 || m.cb == 6) && m.rows >= kSplitMinRows;
}

void dev_free(DeviceSolver& s, void* ptr) {
  if (!ptr) return;
  for (size_t i = 0; i < s.owned.size(); ++i)
    if (s.owned[i].first == ptr) {
      cudaFreeAsync(ptr, s.stream);
      s.bytes -= s.owned[i].second;
      s.owned[i] = s.owned.back();
      s.owned.pop_back();
      return;
    }
}

void dev_free_all(DeviceSolver& s) {
  if (s.graph_exec) cudaGraphExecDestroy(s.graph_exec);
  if (s.graph) cudaGraphDestroy(s.graph);
  s.graph_exec = nullptr;
  s.graph = nullptr;
  for (auto& p : s.owned) cudaFreeAsync(p.first, s.stream);
  s.owned.clear();
  s.bytes = 0;
}

sf_status make_row_groups(DeviceSolver& s, DevBsr& m, const uint32_t* starts, size_t value_bytes) {
  // Rows per group: as many mean rows as fit kGroupTarget bytes (1 to 8, a power of two). The
  // warp splits into that many teams of 32 / teams lanes, one row each, so a warp works on several
  // light rows at once (their x gathers and epilogue loads overlap) and on a heavy row whole.
  double mean = m.rows ? (double)starts[m.rows] / m.rows : 0.0;
  // Batchable studies take a nominal row length per block shape (about 25 blocks on a 3x3
  // stiffness level, 4 on a prolongator, 30 on a coarse level or a transpose), so the choice, and
  // with it the kernel, is the same for every study of that shape.
  if (s.uniform_lanes) mean = (m.rb == 3 && m.cb == 3) ? 25.0 : (m.cb == 6 && m.rb == 3) ? 4.0 : 30.0;
  double row_bytes = std::max(1.0, mean * (double)value_bytes);
  int teams = 1;
  while (teams < 8 && (teams * 2) * row_bytes <= kGroupTarget) teams *= 2;
  m.lanes_per_row = 32 / teams;
  size_t target = std::min<size_t>(kGroupTarget, (size_t)(teams * row_bytes * 1.15));
  std::vector<uint4> g;
  g.reserve(m.rows / 2 + 2);
  uint32_t max_bytes = 0, max_blocks = 0, max_rows = 0;
  uint32_t r = 0;
  while (r < m.rows) {
    uint32_t e = r + 1;
    size_t bytes = (size_t)(starts[e] - starts[r]) * value_bytes;
    while (e < m.rows && bytes + (size_t)(starts[e + 1] - starts[e]) * value_bytes <= target) {
      bytes += (size_t)(starts[e + 1] - starts[e]) * value_bytes;
      ++e;
    }
    max_bytes = std::max<uint32_t>(max_bytes, (uint32_t)bytes);
    max_blocks = std::max<uint32_t>(max_blocks, starts[e] - starts[r]);
    max_rows = std::max<uint32_t>(max_rows, e - r);
    g.push_back(make_uint4(r, e, starts[r], starts[e]));
    r = e;
  }
  m.ngroups = (uint32_t)g.size();
  m.group_bytes = max_bytes;
  m.group_blocks = max_blocks;
  m.group_rows = max_rows;
  if (sf_status e = dev_alloc(s, (void**)&m.groups, std::max<size_t>(1, g.size()) * sizeof(uint4))) return e;
  if (!g.empty()) copy_h2d(s, m.groups, g.data(), g.size() * sizeof(uint4));
  return cuda_check(cudaStreamSynchronize(s.stream), "row groups");
}

namespace {

struct SellLayout {
  uint32_t nslices = 0;
  std::vector<uint32_t> rows, len, start;
};

// Rows by descending block count inside windows of kSellWindow rows, equal lengths in row order:
// a counting sort per window (the order a stable sort by descending length gives).
std::vector<uint32_t> window_order(uint32_t nrows, const uint32_t* starts) {
  std::vector<uint32_t> order(nrows), count;
  for (uint32_t w0 = 0; w0 < nrows; w0 += kSellWindow) {
    const uint32_t w1 = std::min(nrows, w0 + kSellWindow);
    uint32_t longest = 0;
    for (uint32_t r = w0; r < w1; ++r) longest = std::max(longest, starts[r + 1] - starts[r]);
    count.assign(longest + 2, 0);
    for (uint32_t r = w0; r < w1; ++r) count[longest - (starts[r + 1] - starts[r]) + 1] += 1;
    for (uint32_t k = 1; k <= longest + 1; ++k) count[k] += count[k - 1];
    for (uint32_t r = w0; r < w1; ++r) order[w0 + count[longest - (starts[r + 1] - starts[r])]++] = r;
  }
  return order;
}

// Rows sorted by descending block count inside windows of kSellWindow rows (stable, so equal
// lengths keep row order), cut into slices of 32, slice widths padded to chunks of `chunk`
// blocks. Only this row order is host work; the blocks are placed on the device.
SellLayout sell_layout(uint32_t nrows, const uint32_t* starts, uint32_t chunk) {
  SellLayout L;
  L.nslices = (nrows + 31) / 32;
  std::vector<uint32_t> order = window_order(nrows, starts);
  auto rlen = [&](uint32_t r) { return starts[r + 1] - starts[r]; };
  L.rows.assign((size_t)L.nslices * 32, nrows);
  L.len.assign((size_t)L.nslices * 32, 0);
  L.start.assign(L.nslices + 1, 0);
  for (uint32_t i = 0; i < nrows; ++i) {
    L.rows[i] = order[i];
    L.len[i] = rlen(order[i]);
  }
  for (uint32_t sl = 0; sl < L.nslices; ++sl) {
    uint32_t width = 0;
    for (uint32_t t = 0; t < 32; ++t) width = std::max(width, L.len[sl * 32 + t]);
    width = (width + chunk - 1) / chunk * chunk;
    L.start[sl + 1] = L.start[sl] + 32 * width;
  }
  return L;
}

// Block rows ordered as sell_layout orders rows, kSplitRowsPerSlice to a slice, six lanes each
// (lane 6 m + p: scalar row p of the slice's block row m; lanes 30 and 31 idle), slice widths
// padded to chunks of `chunk` blocks.
SellLayout split_layout(uint32_t nrows, const uint32_t* starts, uint32_t chunk) {
  SellLayout L;
  L.nslices = (nrows + kSplitRowsPerSlice - 1) / kSplitRowsPerSlice;
  std::vector<uint32_t> order = window_order(nrows, starts);
  auto rlen = [&](uint32_t r) { return starts[r + 1] - starts[r]; };
  L.rows.assign((size_t)L.nslices * 32, nrows);
  L.len.assign((size_t)L.nslices * 32, 0);
  L.start.assign(L.nslices + 1, 0);
  for (uint32_t i = 0; i < nrows; ++i) {
    const size_t sl = i / kSplitRowsPerSlice, m = i % kSplitRowsPerSlice;
    for (uint32_t p = 0; p < 6; ++p) {
      L.rows[sl * 32 + 6 * m + p] = order[i];
      L.len[sl * 32 + 6 * m + p] = rlen(order[i]);
    }
  }
  for (uint32_t sl = 0; sl < L.nslices; ++sl) {
    uint32_t width = 0;
    for (uint32_t t = 0; t < 32; ++t) width = std::max(width, L.len[sl * 32 + t]);
    width = (width + chunk - 1) / chunk * chunk;
    L.start[sl + 1] = L.start[sl] + 32 * width;
  }
  return L;
}

sf_status upload_sell_layout(DeviceSolver& s, DevBsr& m, const SellLayout& L, size_t value_bytes, bool split) {
  m.nslices = L.nslices;
  sf_status e = SF_OK;
  if (!e) e = dev_alloc(s, (void**)&m.sell_rows, L.rows.size() * 4);
  if (!e) e = dev_alloc(s, (void**)&m.sell_len, L.len.size() * 4);
  if (!e) e = dev_alloc(s, (void**)&m.sell_start, L.start.size() * 4);
  const size_t slots = L.start[L.nslices];
  const size_t col_slots = split ? slots / 32 * kSplitRowsPerSlice : slots;
  if (!e) e = dev_alloc(s, (void**)&m.sell_cols, std::max<size_t>(1, col_slots) * 4);
  if (!e) e = dev_alloc(s, &m.sell_vals, std::max<size_t>(1, slots) * value_bytes);
  if (e) return e;
  copy_h2d(s, m.sell_rows, L.rows.data(), L.rows.size() * 4);
  copy_h2d(s, m.sell_len, L.len.data(), L.len.size() * 4);
  copy_h2d(s, m.sell_start, L.start.data(), L.start.size() * 4);
  return SF_OK;
}

}  // namespace

// The SELL copy of a matrix from its f64 values on the device, converted to S.
template <typename S>
sf_status make_sell_converted(DeviceSolver& s, DevBsr& m, const uint32_t* starts, const uint32_t* cols,
                              const double* vals) {
  const int len = (int)(m.rb * m.cb);
  SellLayout L = sell_layout(m.rows, starts, (uint32_t)sell_chunk_blocks(len, (int)sizeof(S)));
  if (sf_status e = upload_sell_layout(s, m, L, (size_t)len * sizeof(S), false)) return e;
  sf_status e = setup_sell_fill<S>(s.stream, (size_t)L.nslices * 32, len, m.sell_rows, m.sell_len, m.sell_start, m.rows,
                                   m.starts, m.cols, vals, m.sell_cols, (S*)m.sell_vals);
  if (!e) e = cuda_check(cudaStreamSynchronize(s.stream), "SELL placement");
  m.sell = true;
  return e;
}

// The split-row copy of a 6 x cb matrix from its f64 values on the device, converted to S.
template <typename S>
sf_status make_split_converted(DeviceSolver& s, DevBsr& m, const uint32_t* starts, const double* vals) {
  SellLayout L = split_layout(m.rows, starts, (uint32_t)sell_chunk_blocks((int)m.cb, (int)sizeof(S)));
  if (sf_status e = upload_sell_layout(s, m, L, (size_t)m.cb * sizeof(S), true)) return e;
  sf_status e = setup_split_fill<S>(s.stream, (size_t)L.nslices * 32, (int)m.cb, m.sell_rows, m.sell_len, m.sell_start,
                                    m.rows, m.starts, m.cols, vals, m.sell_cols, (S*)m.sell_vals);
  if (!e) e = cuda_check(cudaStreamSynchronize(s.stream), "split-row placement");
  m.split = true;
  return e;
}

sf_status make_sell_from_device(DeviceSolver& s, DevBsr& m, const uint32_t* starts, const uint32_t* cols) {
  (void)cols;
  return make_sell_converted<double>(s, m, starts, nullptr, (const double*)m.vals);
}

namespace {

// A level operator on the device from the setup's f64 values: the setup's device pattern, the
// values converted to S (or the f64 values themselves when S is double and `alias` holds), row
// groups, and a SELL copy when the operator has many rows.
template <typename S>
sf_status device_bsr(DeviceSolver& s, const Bsr& h, DevBsr& d, bool alias) {
  d.rows = (uint32_t)h.rows;
  d.rb = (uint32_t)h.rb;
  d.cb = (uint32_t)h.cb;
  d.blocks = h.cols.size();
  d.starts = h.dev_starts;
  d.cols = h.dev_cols;
  const size_t n = h.cols.size() * h.rb * h.cb;
  if (alias && sizeof(S) == 8) {
    d.vals = h.dev;
  } else {
    if (sf_status e = dev_alloc(s, &d.vals, std::max<size_t>(1, n) * sizeof(S))) return e;
    if (sf_status e = setup_convert<S>(s.stream, n, h.dev, (S*)d.vals)) return e;
  }
  if (sf_status e = make_row_groups(s, d, h.starts.data(), h.rb * h.cb * sizeof(S))) return e;
  if (wants_split(d, s.uniform_lanes)) {
    if (sf_status e = make_split_converted<S>(s, d, h.starts.data(), h.dev)) return e;
  } else if (wants_sell(d, s.sell_min_rows)) {
    if (sf_status e = make_sell_converted<S>(s, d, h.starts.data(), h.cols.data(), h.dev)) return e;
  }
  return cuda_check(cudaGetLastError(), "level operator");
}

// The pattern of a prolongator's explicit transpose (coarse rows, fine block columns ascending)
// and, per transposed block, the prolongator block it comes from (gpu/layout.rs:254-291 stores
// the same transpose for gather restriction).
void transpose_pattern(const Bsr& p, size_t coarse_rows, Bsr& t, std::vector<uint32_t>& src) {
  t = Bsr();
  t.rows = coarse_rows;
  t.rb = p.cb;
  t.cb = p.rb;
  t.starts.assign(coarse_rows + 1, 0);
  for (uint32_t c : p.cols) t.starts[c + 1] += 1;
  for (size_t i = 0; i < coarse_rows; ++i) t.starts[i + 1] += t.starts[i];
  std::vector<uint32_t> fill(t.starts.begin(), t.starts.end() - 1);
  t.cols.resize(p.cols.size());
  src.resize(p.cols.size());
  for (size_t row = 0; row < p.rows; ++row)
    for (uint32_t at = p.starts[row]; at < p.starts[row + 1]; ++at) {
      uint32_t o = fill[p.cols[at]]++;
      t.cols[o] = (uint32_t)row;
      src[o] = at;
    }
}

template <typename S>
sf_status upload_level(DeviceSolver& s, const std::vector<HostLevel>& levels, size_t li, DevLevel& L) {
  const HostLevel& h = levels[li];
  const bool alias = true;
  if (li == 0 && sizeof(S) == 8) {
    L.a = s.system;  // the f64 system matrix is the finest operator
  } else if (sf_status e = device_bsr<S>(s, h.a, L.a, alias)) {
    return e;
  }
  const size_t nd = h.a.rows * h.a.rb * h.a.rb;
  if (sizeof(S) == 8) {
    L.dinv = h.inverse_diagonal;
  } else {
    if (sf_status e = dev_alloc(s, &L.dinv, nd * sizeof(S))) return e;
    if (sf_status e = setup_convert<S>(s.stream, nd, h.inverse_diagonal, (S*)L.dinv)) return e;
  }
  L.has_p = h.has_p;
  if (h.has_p) {
    if (sf_status e = device_bsr<S>(s, h.p, L.p, alias)) return e;
    Bsr t;
    std::vector<uint32_t> src;
    transpose_pattern(h.p, levels[li + 1].a.rows, t, src);
    uint32_t* d_src = nullptr;
    sf_status e = dev_alloc(s, (void**)&d_src, std::max<size_t>(1, src.size()) * 4);
    if (!e) e = dev_alloc(s, (void**)&t.dev_starts, (t.rows + 1) * 4);
    if (!e) e = dev_alloc(s, (void**)&t.dev_cols, std::max<size_t>(1, t.cols.size()) * 4);
    if (!e) e = dev_alloc(s, (void**)&t.dev, std::max<size_t>(1, t.cols.size()) * t.rb * t.cb * 8);
    if (e) return e;
    if (!src.empty()) copy_h2d(s, d_src, src.data(), src.size() * 4);
    copy_h2d(s, t.dev_starts, t.starts.data(), (t.rows + 1) * 4);
    if (!t.cols.empty()) copy_h2d(s, t.dev_cols, t.cols.data(), t.cols.size() * 4);
    e = setup_transpose_blocks<double>(s.stream, t.cols.size(), (int)h.p.rb, (int)h.p.cb, d_src, h.p.dev, t.dev);
    if (!e) e = device_bsr<S>(s, t, L.r, alias);
    if (!e) e = cuda_check(cudaStreamSynchronize(s.stream), "transpose");
    dev_free(s, d_src);
    if (sizeof(S) != 8) dev_free(s, t.dev);  // the converted copy is the one kept
    if (e) return e;
  }
  return SF_OK;
}

}  // namespace

sf_status solver_upload_hierarchy(DeviceSolver& s, const std::vector<HostLevel>& levels, uint64_t degree) {
  size_t V = s.vector_single ? 4 : 8;
  s.levels.assign(levels.size(), DevLevel());
  for (size_t li = 0; li < levels.size(); ++li) {
    const HostLevel& h = levels[li];
    DevLevel& L = s.levels[li];
    L.n = (uint32_t)(h.a.rows * h.a.rb);
    sf_status e = s.storage_single ? upload_level<float>(s, levels, li, L) : upload_level<double>(s, levels, li, L);
    if (e) return e;
    L.has_factor = h.has_factor;
    if (h.has_factor) {
      L.coarse_inverse = h.dev_coarse_inverse;  // made on the device by the setup, owned by this solver
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
  // The coarse tail: the last smoothed level (6-row blocks) and the factored coarsest level,
  // small enough that one cluster beats a launch per phase. Batchable studies keep per-phase
  // launches (their kernel sequence must not depend on sizes).
  s.tail_level = -1;
  s.tail_cluster = 0;
  s.tail_smem = 0;
  if (s.coarse_tail && !s.uniform_lanes && s.levels.size() >= 3) {
    const size_t li = s.levels.size() - 2;
    const DevLevel& L = s.levels[li];
    const DevLevel& C = s.levels[li + 1];
    if (L.has_p && C.has_factor && L.a.rb == 6 && L.a.cb == 6 && L.p.rb == 6 && L.p.cb == 6 && L.r.rb == 6 &&
        L.r.cb == 6 && L.a.rows <= kTailMaxRows && C.n <= kTailMaxCoarse && L.steps.size() <= (size_t)kTailMaxSteps) {
      size_t smem = 0;
      const HostLevel &hs = levels[li], &hc = levels[li + 1];
      unsigned c = !s.storage_single ? tail_cluster_size<double, double>(hs, hc, &smem)
                   : !s.vector_single ? tail_cluster_size<float, double>(hs, hc, &smem)
                                      : tail_cluster_size<float, float>(hs, hc, &smem);
      if (c) {
        s.tail_level = (int)li;
        s.tail_cluster = c;
        s.tail_smem = smem;
      }
    }
  }
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
  launch_body<pcg_init_kernel>(kReduceBlocks, kReduceThreads, 0, s.stream, s.n, s.rhs, s.x, s.r, s.partials, s.state);
  return solver_enqueue_reset(s);
}

sf_status solver_enqueue_reset(DeviceSolver& s) {
  const int* status = &s.state->status;
  enqueue_precondition(s, s.r, s.z, s.z32, status);
  if (s.vector_single && s.multigrid) {
    launch_body<pcg_dot_rz_kernel<float>>(kReduceBlocks, kReduceThreads, 0, s.stream, s.n, s.r, s.z32, s.ap, s.partials, s.state);
    launch_body<pcg_update_p_kernel<float>>(grid_for_elems(s.n), kThreads, 0, s.stream, s.n, s.z32, s.p, s.state);
  } else {
    launch_body<pcg_dot_rz_kernel<double>>(kReduceBlocks, kReduceThreads, 0, s.stream, s.n, s.r, s.z, s.ap, s.partials, s.state);
    launch_body<pcg_update_p_kernel<double>>(grid_for_elems(s.n), kThreads, 0, s.stream, s.n, s.z, s.p, s.state);
  }
  s.launches_per_iteration += 2;
  return cuda_check(cudaGetLastError(), "reset direction");
}

sf_status solver_enqueue_iteration(DeviceSolver& s) {
  cudaStream_t st = s.stream;
  const int* status = &s.state->status;
  s.launches_per_iteration = 0;
  if (s.system.sell) {
    SellOp<double> A = sell_of<double>(s.system);
    int grid = std::min(grid_for_slices(s.system.nslices), kReduceBlocks * 2);
    launch_body<sell_pcg_spmv_dot_kernel>(grid, kThreads, 0, st, A, s.p, s.ap, s.partials, s.state);
    launch_body<pcg_update_kernel>(kReduceBlocks, kReduceThreads, 0, st, s.n, s.p, s.ap, s.x, s.r, s.partials, s.state);
    launch_body<sell_pcg_check_kernel>(grid, kThreads, 0, st, A, s.x, s.rhs, s.r, s.partials, s.state);
  } else switch (s.system.lanes_per_row) {
    case 8: launch_pcg_spmv_lpr<8>(s); break;
    case 16: launch_pcg_spmv_lpr<16>(s); break;
    default: launch_pcg_spmv_lpr<32>(s); break;
  }
  s.launches_per_iteration += 3;
  enqueue_precondition(s, s.r, s.z, s.z32, status);
  if (s.vector_single && s.multigrid) {
    launch_body<pcg_dot_rz_kernel<float>>(kReduceBlocks, kReduceThreads, 0, st, s.n, s.r, s.z32, s.ap, s.partials, s.state);
    launch_body<pcg_update_p_kernel<float>>(grid_for_elems(s.n), kThreads, 0, st, s.n, s.z32, s.p, s.state);
  } else {
    launch_body<pcg_dot_rz_kernel<double>>(kReduceBlocks, kReduceThreads, 0, st, s.n, s.r, s.z, s.ap, s.partials, s.state);
    launch_body<pcg_update_p_kernel<double>>(grid_for_elems(s.n), kThreads, 0, st, s.n, s.z, s.p, s.state);
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

// ------------------------------------------------------------ batched iterations
// Records one conjugate gradient iteration of every instance, checks that they launch the same
// kernels in the same order with the same block shapes, and captures one graph whose every node
// is a single grid over all instances: grid.x is the largest instance's, grid.y the instance
// count, and each launch site's argument packs sit in one device table (the per-instance offset
// table: each pack holds that instance's operator, vectors, scalars and status word).
sf_status batch_build(const std::vector<DeviceSolver*>& inst, cudaStream_t stream, BatchIteration& out) {
  out = BatchIteration();
  out.stream = stream;
  out.count = inst.size();
  if (inst.empty()) return fail(SF_INVALID_ARGUMENT, "an empty batch");
  std::vector<std::vector<LaunchRecord>> rec(inst.size());
  for (size_t i = 0; i < inst.size(); ++i) {
    g_recorder = &rec[i];
    sf_status e = solver_enqueue_iteration(*inst[i]);
    g_recorder = nullptr;
    if (e) return e;
  }
  const size_t sites = rec[0].size();
  for (size_t i = 1; i < inst.size(); ++i) {
    const char* why = nullptr;
    size_t at = 0;
    if (rec[i].size() != sites) why = "a different number of kernels per iteration";
    for (size_t j = 0; !why && j < sites; ++j) {
      at = j;
      if (rec[i][j].batched != rec[0][j].batched) why = "a different kernel";
      else if (rec[i][j].pack.size() != rec[0][j].pack.size()) why = "different arguments";
      else if (rec[i][j].cluster != rec[0][j].cluster) why = "a different cluster size";
    }
    if (why) {
      char msg[200];
      std::snprintf(msg, sizeof msg, "the studies of a batch must share their launch structure: study %zu has %s (launch %zu)",
                    i, why, at);
      return fail(SF_INVALID_ARGUMENT, msg);
    }
  }
  struct Site {
    const void* kernel;
    dim3 grid, block;
    size_t smem;
    void* table;
    unsigned cluster;
  };
  std::vector<Site> list(sites);
  for (size_t j = 0; j < sites; ++j) {
    Site& t = list[j];
    t.kernel = rec[0][j].batched;
    t.block = rec[0][j].block;
    t.grid = dim3(1, (unsigned)inst.size(), 1);
    t.smem = 0;
    t.cluster = rec[0][j].cluster;
    const size_t bytes = rec[0][j].pack.size();
    std::vector<unsigned char> host(bytes * inst.size());
    // Block sizes may differ (a row-group kernel's warps per block follow its largest group); the
    // bodies work with any block size and place each warp's staging slot by their own operator,
    // so the batch takes the largest block and the largest per-warp slot.
    size_t per_warp = 0;
    for (size_t i = 0; i < inst.size(); ++i) {
      t.grid.x = std::max(t.grid.x, rec[i][j].grid.x);
      t.block.x = std::max(t.block.x, rec[i][j].block.x);
      per_warp = std::max(per_warp, rec[i][j].smem / std::max(1u, rec[i][j].block.x / 32));
      if (t.cluster) t.smem = std::max(t.smem, rec[i][j].smem);
      std::memcpy(host.data() + i * bytes, rec[i][j].pack.data(), bytes);
    }
    if (t.cluster) {
      // a cluster kernel keeps its block (launch bounds) and the largest instance's shared memory
    } else if (per_warp > 0) {
      // Fewer warps per block when the largest slot would not fit 200 KB of shared memory.
      size_t warps = std::max<size_t>(1, std::min<size_t>(t.block.x / 32, (200 * 1024) / per_warp));
      t.block.x = (unsigned)(32 * warps);
    }
    if (!t.cluster) t.smem = per_warp * (t.block.x / 32);
    if (t.smem > 200 * 1024) {
      batch_destroy(out);
      return fail(SF_INVALID_ARGUMENT, "a study of the batch needs more shared memory per warp than one SM holds");
    }
    pool_setup(inst[0]->device);
    cudaError_t e = cudaMallocAsync(&t.table, std::max<size_t>(host.size(), 16), stream);
    if (e != cudaSuccess) {
      batch_destroy(out);
      return cuda_check(e, "batch table");
    }
    out.tables.push_back(t.table);
    e = cudaMemcpyAsync(t.table, host.data(), host.size(), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess && t.smem > 48 * 1024)
      e = cudaFuncSetAttribute(t.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e != cudaSuccess) {
      batch_destroy(out);
      return cuda_check(e, "batch table");
    }
  }
  out.sites = sites;
  cudaError_t e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    batch_destroy(out);
    return cuda_check(e, "begin batch capture");
  }
  cudaError_t launch = cudaSuccess;
  for (Site& t : list) {
    cudaLaunchAttribute attr[1];
    if (t.cluster) {
      // one cluster per instance: grid.x is the cluster, blockIdx.y the instance
      t.grid.x = t.cluster;
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = t.cluster;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
    } else {
      attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      attr[0].val.programmaticStreamSerializationAllowed = 1;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = t.grid;
    cfg.blockDim = t.block;
    cfg.dynamicSmemBytes = t.smem;
    cfg.stream = stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void* argv[1] = {&t.table};
    cudaError_t le = cudaLaunchKernelExC(&cfg, t.kernel, argv);
    if (le != cudaSuccess && launch == cudaSuccess) launch = le;
  }
  e = cudaStreamEndCapture(stream, &out.graph);
  if (launch != cudaSuccess || e != cudaSuccess) {
    batch_destroy(out);
    return cuda_check(launch != cudaSuccess ? launch : e, "batch capture");
  }
  e = cudaGraphInstantiate(&out.exec, out.graph, 0);
  if (e != cudaSuccess) {
    batch_destroy(out);
    return cuda_check(e, "batch instantiate");
  }
  return SF_OK;
}

sf_status batch_replay(BatchIteration& b, uint64_t iterations) {
  for (uint64_t i = 0; i < iterations; ++i) {
    cudaError_t e = cudaGraphLaunch(b.exec, b.stream);
    if (e != cudaSuccess) return cuda_check(e, "batch replay");
  }
  return SF_OK;
}

void batch_destroy(BatchIteration& b) {
  if (b.exec) cudaGraphExecDestroy(b.exec);
  if (b.graph) cudaGraphDestroy(b.graph);
  for (void* t : b.tables) cudaFreeAsync(t, b.stream);
  b.exec = nullptr;
  b.graph = nullptr;
  b.tables.clear();
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

namespace {

// One stage of level li's V-cycle on the level's own buffers, through the launches the cycle
// makes (same layouts, same fused epilogues): inputs in f64 device memory are rounded to the
// vector type first, outputs widened to f64. The stages and their buffers:
//   SMOOTH          b -> L.b;  smoother from zero into L.x
//   SMOOTH_ADD      b -> L.b, x -> L.tmp;  L.tmp += smoother (the post-smoother's last step)
//   START           b -> L.b;  the start kernel: L.x = (D^-1 b) / theta
//   RESIDUAL        b -> L.b, x -> L.x;  L.res = b - A x
//   RESTRICT        r -> L.res;  C.b = R r
//   PROLONG         e -> C.x, x -> L.x;  L.x += P e
//   RESTRICT_START  r -> L.res;  C.b = R r with the coarser level's start fused in (C.x)
//   RESIDUAL_START  b -> L.b, x -> L.x;  L.res = b - A x with the start fused in (L.post_x)
template <typename S, typename V>
sf_status level_stage(DeviceSolver& s, size_t li, int stage, const double* in0, const double* in1, double* out0,
                      double* out1) {
  DevLevel& L = s.levels[li];
  const bool coarse = li + 1 < s.levels.size();
  DevLevel* C = coarse ? &s.levels[li + 1] : nullptr;
  cudaStream_t st = s.stream;
  const int* on = s.always_active;
  auto to_v = [&](const double* src, void* dst, uint32_t n) {
    launch_body<convert_kernel<double, V>>(grid_for_elems(n), kThreads, 0, st, n, src, (V*)dst, on);
  };
  auto from_v = [&](const void* src, double* dst, uint32_t n) {
    launch_body<convert_kernel<V, double>>(grid_for_elems(n), kThreads, 0, st, n, (const V*)src, dst, on);
  };
  const bool smoothed = L.has_p || !L.has_factor;
  switch (stage) {
    case SF_STAGE_SMOOTH:
    case SF_STAGE_SMOOTH_ADD:
    case SF_STAGE_START:
      if (!smoothed) return fail(SF_INVALID_ARGUMENT, "the coarsest level is factored, not smoothed");
      to_v(in0, L.b, L.n);
      if (stage == SF_STAGE_START) {
        if (L.a.rb == 3)
          launch_cheb_start<S, V, V, 3>(L, (const V*)L.b, nullptr, (V*)L.res, (V*)L.d0, (V*)L.x, L.theta, on, st);
        else
          launch_cheb_start<S, V, V, 6>(L, (const V*)L.b, nullptr, (V*)L.res, (V*)L.d0, (V*)L.x, L.theta, on, st);
        from_v(L.x, out0, L.n);
      } else if (stage == SF_STAGE_SMOOTH) {
        enqueue_smooth<S, V, V>(s, L, (const V*)L.b, nullptr, (V*)L.x, nullptr, on);
        from_v(L.x, out0, L.n);
      } else {
        to_v(in1, L.tmp, L.n);
        enqueue_smooth<S, V, V>(s, L, (const V*)L.b, nullptr, (V*)L.post_x, (V*)L.tmp, on);
        from_v(L.tmp, out0, L.n);
      }
      break;
    case SF_STAGE_RESIDUAL:
    case SF_STAGE_RESIDUAL_START:
      to_v(in0, L.b, L.n);
      to_v(in1, L.x, L.n);
      if (stage == SF_STAGE_RESIDUAL) {
        bsr_dispatch<S, V, OP_RESIDUAL>(L.a, (const V*)L.x, (V*)L.res, (const V*)L.b, on, st);
      } else {
        if (!smoothed) return fail(SF_INVALID_ARGUMENT, "the coarsest level is factored, not smoothed");
        launch_start_product<S, V, OP_RESIDUAL>(L.a, (const V*)L.x, (const V*)L.b,
                                                start_args<S, V>(L, (V*)nullptr, (V*)L.post_x), on, st);
        from_v(L.post_x, out1, L.n);
      }
      from_v(L.res, out0, L.n);
      break;
    case SF_STAGE_RESTRICT:
    case SF_STAGE_RESTRICT_START:
      if (!L.has_p) return fail(SF_INVALID_ARGUMENT, "the level has no coarser level");
      to_v(in0, L.res, L.n);
      if (stage == SF_STAGE_RESTRICT) {
        bsr_dispatch<S, V, OP_SET>(L.r, (const V*)L.res, (V*)C->b, nullptr, on, st);
      } else {
        if (!C->has_p && C->has_factor) return fail(SF_INVALID_ARGUMENT, "the coarser level is factored, not smoothed");
        launch_start_product<S, V, OP_SET>(L.r, (const V*)L.res, (const V*)nullptr,
                                           start_args<S, V>(*C, (V*)C->b, (V*)C->x), on, st);
        from_v(C->x, out1, C->n);
      }
      from_v(C->b, out0, C->n);
      break;
    case SF_STAGE_PROLONG:
      if (!L.has_p) return fail(SF_INVALID_ARGUMENT, "the level has no coarser level");
      to_v(in0, C->x, C->n);
      to_v(in1, L.x, L.n);
      bsr_dispatch<S, V, OP_ADD>(L.p, (const V*)C->x, (V*)L.x, nullptr, on, st);
      from_v(L.x, out0, L.n);
      break;
    default:
      return fail(SF_INVALID_ARGUMENT, "unknown stage");
  }
  s.launches += 4;
  return cuda_check(cudaStreamSynchronize(st), "level stage");
}

}  // namespace

sf_status solver_level_stage(DeviceSolver& s, size_t level, int stage, const double* in0, const double* in1,
                             double* out0, double* out1) {
  if (!s.multigrid || level >= s.levels.size()) return fail(SF_INVALID_ARGUMENT, "no such multigrid level");
  if (!s.storage_single) return level_stage<double, double>(s, level, stage, in0, in1, out0, out1);
  if (!s.vector_single) return level_stage<float, double>(s, level, stage, in0, in1, out0, out1);
  return level_stage<float, float>(s, level, stage, in0, in1, out0, out1);
}

sf_status solver_precondition(DeviceSolver& s, const double* d_in, double* d_out) {
  enqueue_precondition(s, d_in, d_out, s.z32, s.always_active);
  if (s.vector_single && s.multigrid)
    launch_body<convert_kernel<float, double>>(grid_for_elems(s.n), kThreads, 0, s.stream, s.n, s.z32, d_out, s.always_active);
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

// ------------------------------------------------------------ energy products, allocating nothing
// A variant of the conjugate gradient's system product (pcg_spmv_dot_kernel and
// sell_pcg_spmv_dot_kernel): for each of `count` vectors x_k of caller-owned device memory it
// writes y_k = A x_k and the energy e_k = x_k . y_k. Rows are summed exactly as the system product
// sums them; vector k runs in blockIdx.y = k. The reduction's scratch is not the solver's: it is
// the file-scope array below, whose address is looked up once per device, so a call allocates no
// memory at all.
//
// Scratch layout (g_energy_scratch, 65,792 bytes per device):
//   bytes [0, 256):   one arrival ticket (unsigned) per vector. Each ticket must be zero when a
//                     launch starts. Static device storage is zero when the module loads, and the
//                     last block of each vector puts its ticket back to zero before it exits, so
//                     the tickets are zero again after every completed call.
//   bytes [256, ...): kEnergyMaxBlocks partial sums per vector. No initial value is needed: every
//                     block writes its slot before it takes its ticket.
// One array serves every study on a device, so two calls whose kernels can run at the same time
// (different streams, different studies, different host threads) race on it.
constexpr int kEnergyMaxVectors = 8;
constexpr int kEnergyMaxBlocks = 1024;  // blocks per vector of one launch
constexpr size_t kEnergyTicketBytes = 256;
constexpr size_t kEnergyScratchBytes = kEnergyTicketBytes + (size_t)kEnergyMaxVectors * kEnergyMaxBlocks * sizeof(double);
constexpr int kEnergyMaxDevices = 64;
static_assert(kEnergyMaxVectors * sizeof(unsigned) <= kEnergyTicketBytes, "tickets fit their header");

static __device__ __align__(256) unsigned char g_energy_scratch[kEnergyScratchBytes];

namespace {

__device__ __forceinline__ void energy_finish(double local, unsigned char* scratch, double* energy) {
  const uint32_t k = blockIdx.y;
  unsigned* tickets = reinterpret_cast<unsigned*>(scratch);
  double* partials = reinterpret_cast<double*>(scratch + kEnergyTicketBytes) + (size_t)k * kEnergyMaxBlocks;
  double v[1] = {local}, total[1];
  if (finish_partials<1>(v, partials, tickets + k, total) && threadIdx.x == 0) energy[k] = total[0];
}

// SELL-32 system: one thread per row, rows summed as sell_kernel sums them.
__global__ void __launch_bounds__(kThreads) sell_energy_kernel(SellOp<double> A, const double* __restrict__ x,
                                                                double* __restrict__ y, uint32_t n,
                                                                double* __restrict__ energy, unsigned char* scratch) {
  const size_t off = (size_t)blockIdx.y * n;
  SellDot epi;
  epi.p = x + off;
  epi.ap = y + off;
  epi.local = 0.0;
  sell_rows<double, double, 3, 3, false>(A, x + off, epi, OpenGate{});
  energy_finish(epi.local, scratch, energy);
}

// Row-group system: LPR lanes per row, rows summed as bsr_kernel sums them.
template <int LPR>
__global__ void __launch_bounds__(kThreads) energy_kernel(Op<double> A, const double* __restrict__ x,
                                                           double* __restrict__ y, uint32_t n,
                                                           double* __restrict__ energy, unsigned char* scratch) {
  extern __shared__ __align__(16) char smem[];
  char* wbase = smem + (threadIdx.x >> 5) * 2 * slot_bytes(A);
  const size_t off = (size_t)blockIdx.y * n;
  EpiDot<LPR> epi;
  epi.p = x + off;
  epi.ap = y + off;
  epi.local = 0.0;
  run_groups<double, double, 3, 3, LPR, false>(A, x + off, wbase, epi, OpenGate{});
  energy_finish(epi.local, scratch, energy);
}

std::mutex g_energy_mutex;
unsigned char* g_energy_address[kEnergyMaxDevices] = {};

// Once per device, with that device current: the scratch's device address and the row-group
// variants' shared-memory opt-in. Neither allocates memory; the first lookup on a device can load
// this library's device code there.
sf_status energy_setup(int device, unsigned char** out) {
  std::lock_guard<std::mutex> lock(g_energy_mutex);
  if (device < 0 || device >= kEnergyMaxDevices) return fail(SF_INVALID_ARGUMENT, "device ordinal out of range");
  if (!g_energy_address[device]) {
    unsigned char* ptr = nullptr;
    if (sf_status e = cuda_check(cudaGetSymbolAddress((void**)&ptr, g_energy_scratch), "cudaGetSymbolAddress"))
      return e;
    const int smem = 200 * 1024;
    cudaError_t e = cudaFuncSetAttribute(energy_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(energy_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(energy_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(energy_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (sf_status st = cuda_check(e, "cudaFuncSetAttribute")) return st;
    g_energy_address[device] = ptr;
  }
  *out = g_energy_address[device];
  return SF_OK;
}

template <int LPR>
void launch_energy_lpr(const DevBsr& m, const double* x, double* y, uint32_t n, double* energy, uint64_t count,
                       unsigned char* scratch, cudaStream_t st) {
  Op<double> A = op_of<double>(m);
  Shape sh = shape_of(A, true);
  dim3 grid((unsigned)std::min(sh.grid, kEnergyMaxBlocks), (unsigned)count);
  energy_kernel<LPR><<<grid, sh.threads, sh.smem, st>>>(A, x, y, n, energy, scratch);
}

}  // namespace

uint64_t solver_energy_max_vectors() { return kEnergyMaxVectors; }

sf_status solver_energy_products(DeviceSolver& s, const double* x, double* y, double* energy, uint64_t count) {
  if (count > (uint64_t)kEnergyMaxVectors) {
    char msg[160];
    std::snprintf(msg, sizeof msg, "count %llu exceeds the %d vectors the energy scratch holds",
                  (unsigned long long)count, kEnergyMaxVectors);
    return fail(SF_INVALID_ARGUMENT, msg);
  }
  if (count == 0) return SF_OK;
  unsigned char* scratch = nullptr;
  if (sf_status e = energy_setup(s.device, &scratch)) return e;
  const DevBsr& m = s.system;
  if (m.sell) {
    SellOp<double> A = sell_of<double>(m);
    dim3 grid((unsigned)std::min(grid_for_slices(m.nslices), kEnergyMaxBlocks), (unsigned)count);
    sell_energy_kernel<<<grid, kThreads, 0, s.stream>>>(A, x, y, s.n, energy, scratch);
  } else {
    switch (m.lanes_per_row) {
      case 4: launch_energy_lpr<4>(m, x, y, s.n, energy, count, scratch, s.stream); break;
      case 8: launch_energy_lpr<8>(m, x, y, s.n, energy, count, scratch, s.stream); break;
      case 16: launch_energy_lpr<16>(m, x, y, s.n, energy, count, scratch, s.stream); break;
      default: launch_energy_lpr<32>(m, x, y, s.n, energy, count, scratch, s.stream); break;
    }
  }
  s.launches += 1;
  return cuda_check(cudaGetLastError(), "energy products");
}

}  // namespace sf
