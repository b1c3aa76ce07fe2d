// Raw systems: the solver crate's own seam (crates/solidfem-solve). A symmetric matrix given as
// scalar CSR (CsrMatrix, csr.rs:6-13) with a right-hand side, solved on the device by the
// conjugate gradient (Pcg, pcg.rs:133-301) under the Jacobi preconditioner
// (preconditioner.rs:49-79) or the block smoothed-aggregation multigrid
// (MultigridSetup::new / step / finish, multigrid/setup.rs:129-215). Studies reach the same device
// solver through assembly; this entry takes the matrix directly, as the reference's solver tests
// and benches do.
//
// The device kernels work on 3x3 blocks. A multigrid system must already be nodal (rows in threes
// sharing whole three-column blocks: BlockCsr::from_nodal, block.rs:51-99), as the reference
// requires. A Jacobi system of any size is laid out in 3x3 blocks over ceil(n / 3) block rows;
// the padding unknowns (when n is not a multiple of 3) carry an identity row and a zero
// right-hand side, so their residual, preconditioned residual and direction stay exactly zero and
// every dot product and row sum of the real unknowns is the one of the unpadded system.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "device.h"
#include "sf_internal.h"

using namespace sf;
using std::vector;

struct sf_system {
  sf_study_options options;
  uint64_t n = 0;                 // the caller's unknowns
  vector<uint32_t> starts, cols;  // the 3x3 block pattern
  DeviceSolver solver;
  vector<HostLevel> levels;
  int status = ST_ACTIVE;
  bool cancelled = false;
  PcgState last{};
  PcgState* pinned = nullptr;
  ~sf_system() {
    pinned_release(pinned);
    dev_free_all(solver);
    if (solver.stream) cudaStreamDestroy(solver.stream);
  }
};

namespace {

sf_status refuse(const char* message) { return fail(SF_INVALID_ARGUMENT, message); }

// A well-formed CSR matrix: row_starts ascending from 0, columns below n and strictly ascending
// within each row (the invariant every CsrMatrix constructor keeps, csr.rs:19-71).
sf_status check_csr(uint64_t n, const uint64_t* row_starts, const uint32_t* columns) {
  if (row_starts[0] != 0) return refuse("row_starts[0] must be 0");
  for (uint64_t r = 0; r < n; ++r) {
    if (row_starts[r + 1] < row_starts[r]) {
      error_slot().row = r;
      return refuse("row_starts must not decrease");
    }
    for (uint64_t k = row_starts[r]; k < row_starts[r + 1]; ++k) {
      if (columns[k] >= n || (k > row_starts[r] && columns[k] <= columns[k - 1])) {
        error_slot().row = r;
        return refuse("each row's columns must be below n and strictly ascending");
      }
    }
  }
  return SF_OK;
}

// BlockCsr::from_nodal (block.rs:51-99): the rows of each node share one pattern of whole,
// aligned three-column blocks; the first row that breaks it is named.
sf_status from_nodal(uint64_t n, const uint64_t* rs, const uint32_t* cols, const double* vals, vector<uint32_t>& starts,
                     vector<uint32_t>& bcols, vector<double>& bvals) {
  if (n % 3 != 0) {
    error_slot().row = n;
    return fail(SF_MG_BLOCK_STRUCTURE, "the matrix does not group into 3x3 blocks");
  }
  const uint64_t rows = n / 3;
  starts.assign(1, 0);
  for (uint64_t node = 0; node < rows; ++node) {
    const uint64_t r0 = 3 * node;
    const uint64_t len = rs[r0 + 1] - rs[r0];
    for (int q = 1; q < 3; ++q) {
      const uint64_t rq = r0 + q;
      bool same = rs[rq + 1] - rs[rq] == len &&
                  std::equal(cols + rs[r0], cols + rs[r0 + 1], cols + rs[rq]);
      if (!same) {
        error_slot().row = rq;
        return fail(SF_MG_BLOCK_STRUCTURE, "the matrix does not group into 3x3 blocks");
      }
    }
    if (len % 3 != 0) {
      error_slot().row = r0;
      return fail(SF_MG_BLOCK_STRUCTURE, "the matrix does not group into 3x3 blocks");
    }
    const uint32_t* c = cols + rs[r0];
    for (uint64_t at = 0; at < len; at += 3) {
      if (c[at] % 3 != 0 || c[at + 1] != c[at] + 1 || c[at + 2] != c[at] + 2) {
        error_slot().row = r0;
        return fail(SF_MG_BLOCK_STRUCTURE, "the matrix does not group into 3x3 blocks");
      }
      bcols.push_back(c[at] / 3);
      for (int p = 0; p < 3; ++p)
        for (int q = 0; q < 3; ++q) bvals.push_back(vals[rs[r0 + p] + at + q]);
    }
    starts.push_back((uint32_t)bcols.size());
  }
  return SF_OK;
}

// Any scalar matrix over ceil(n / 3) block rows: the blocks its entries touch (and the last
// diagonal block when padding rows are added), zeros where it has no entry, identity on the
// padding's diagonal.
void padded_blocks(uint64_t n, const uint64_t* rs, const uint32_t* cols, const double* vals, vector<uint32_t>& starts,
                   vector<uint32_t>& bcols, vector<double>& bvals) {
  const uint64_t rows = (n + 2) / 3;
  starts.assign(1, 0);
  vector<uint32_t> mark(rows, UINT32_MAX);
  vector<uint32_t> row_cols;
  for (uint64_t b = 0; b < rows; ++b) {
    row_cols.clear();
    for (uint64_t r = 3 * b; r < std::min<uint64_t>(3 * b + 3, n); ++r)
      for (uint64_t k = rs[r]; k < rs[r + 1]; ++k) {
        uint32_t c = cols[k] / 3;
        if (mark[c] != b) {
          mark[c] = (uint32_t)b;
          row_cols.push_back(c);
        }
      }
    if (3 * b + 3 > n && mark[b] != b) row_cols.push_back((uint32_t)b);
    std::sort(row_cols.begin(), row_cols.end());
    const size_t first = bcols.size();
    bcols.insert(bcols.end(), row_cols.begin(), row_cols.end());
    bvals.resize(bcols.size() * 9, 0.0);
    for (int p = 0; p < 3; ++p) {
      const uint64_t r = 3 * b + p;
      if (r >= n) {  // padding: a decoupled identity row
        size_t at = std::lower_bound(bcols.begin() + first, bcols.end(), (uint32_t)b) - bcols.begin();
        bvals[at * 9 + p * 3 + p] = 1.0;
        continue;
      }
      size_t at = first;
      for (uint64_t k = rs[r]; k < rs[r + 1]; ++k) {
        const uint32_t c = cols[k] / 3;
        while (bcols[at] != c) ++at;
        bvals[at * 9 + p * 3 + cols[k] % 3] = vals[k];
      }
    }
    starts.push_back((uint32_t)bcols.size());
  }
}

}  // namespace

extern "C" {

sf_status sf_system_create(uint64_t n, const uint64_t* row_starts, const uint32_t* columns, const double* values,
                           const double* rhs, const double* near_null, uint64_t near_null_count,
                           const double* positions, uint64_t position_count, const sf_study_options* options,
                           sf_cancel_fn cancel, void* user, sf_system** out) {
  if (!out) return refuse("null output");
  *out = nullptr;
  if (!row_starts || !rhs || (n && (!columns || !values))) return refuse("null argument");
  if (n == 0) return refuse("an empty system");
  if (n >= (uint64_t)UINT32_MAX / 2) return refuse("too many unknowns for 32-bit column indices");
  if (sf_status e = check_csr(n, row_starts, columns)) return e;
  std::unique_ptr<sf_system> sys(new sf_system);
  if (options) {
    sys->options = *options;
  } else {
    sf_study_options_default(&sys->options);
  }
  const sf_study_options& o = sys->options;
  const bool mg = o.preconditioner == SF_PRECONDITIONER_MULTIGRID;
  sys->n = n;
  vector<double> bvals;
  if (mg) {
    // MultigridSetup::new (setup.rs:129-160): the near-null length, the nodal blocks, then the
    // positions, each refused by name.
    if (near_null_count != 6 * n || !near_null) {
      error_slot().expected = 6 * n;
      error_slot().found = near_null ? near_null_count : 0;
      return fail(SF_MG_NEAR_NULL_LENGTH, "the near-null space needs six values per unknown");
    }
    if (sf_status e = from_nodal(n, row_starts, columns, values, sys->starts, sys->cols, bvals)) return e;
    if (position_count != n / 3 || !positions) {
      error_slot().expected = n / 3;
      error_slot().found = positions ? position_count : 0;
      return fail(SF_MG_POSITION_LENGTH, "positions need one point per block row");
    }
  } else {
    // Jacobi::new (preconditioner.rs:49-79): a positive, finite diagonal.
    for (uint64_t r = 0; r < n; ++r) {
      const uint32_t* lo = columns + row_starts[r];
      const uint32_t* hi = columns + row_starts[r + 1];
      const uint32_t* at = std::lower_bound(lo, hi, (uint32_t)r);
      const double v = at != hi && *at == r ? values[at - columns] : 0.0;
      if (std::isnan(v) || v <= 0.0 || !std::isfinite(v)) {
        error_slot().row = r;
        error_slot().value = v;
        return fail(SF_JACOBI_DIAGONAL, "a diagonal entry is not positive");
      }
    }
    padded_blocks(n, row_starts, columns, values, sys->starts, sys->cols, bvals);
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(SF_NO_DEVICE, "no CUDA device is visible");
  if (o.device < 0 || o.device >= ndev) return refuse("no such CUDA device");
  cudaSetDevice(o.device);
  DeviceSolver& d = sys->solver;
  d.device = o.device;
  d.sell_min_rows = o.sell_min_rows ? o.sell_min_rows : 32768;
  d.coarse_tail = o.coarse_tail != 0;
  if (sf_status e = cuda_check(cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking), "stream")) return e;
  const size_t rows = sys->starts.size() - 1, blocks = sys->cols.size();
  d.n = (uint32_t)(3 * rows);
  d.system.rows = (uint32_t)rows;
  d.system.rb = d.system.cb = 3;
  d.system.blocks = blocks;
  sf_status e = SF_OK;
  if (!e) e = dev_alloc(d, (void**)&d.system.starts, (rows + 1) * 4);
  if (!e) e = dev_alloc(d, (void**)&d.system.cols, std::max<size_t>(1, blocks) * 4);
  if (!e) e = dev_alloc(d, &d.system.vals, std::max<size_t>(1, blocks) * 72);
  if (e) return e;
  copy_h2d(d, d.system.starts, sys->starts.data(), (rows + 1) * 4);
  if (blocks) {
    copy_h2d(d, d.system.cols, sys->cols.data(), blocks * 4);
    copy_h2d(d, d.system.vals, bvals.data(), blocks * 72);
  }
  if ((e = make_row_groups(d, d.system, sys->starts.data(), 72))) return e;
  if ((e = cuda_check(cudaStreamSynchronize(d.stream), "system upload"))) return e;
  d.multigrid = mg;
  const int prec = o.precision;
  d.precision = prec;
  d.storage_single = mg && prec != SF_PRECISION_DOUBLE;
  d.vector_single = mg && (prec == SF_PRECISION_SINGLE || prec == SF_PRECISION_MIXED);
  d.flexible = mg && prec == SF_PRECISION_MIXED;
  if (mg) {
    Bsr fine;
    fine.rows = rows;
    fine.rb = fine.cb = 3;
    fine.starts = sys->starts;
    fine.cols = sys->cols;
    fine.dev = (double*)d.system.vals;
    fine.dev_starts = d.system.starts;
    fine.dev_cols = d.system.cols;
    vector<double> modes(near_null, near_null + near_null_count);
    vector<P3> pos(rows);
    for (size_t i = 0; i < rows; ++i) pos[i] = {positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]};
    SetupOptions so;
    so.reach = o.neighbour_reach;
    so.coarse_dofs = o.coarse_dofs;
    so.max_levels = o.max_levels;
    so.range = o.smoother_range;
    so.threads = o.threads ? (int)std::min<uint64_t>(o.threads, 64) : default_threads();
    SetupMachine* machine = setup_create(d, std::move(fine), std::move(modes), std::move(pos), so);
    bool finished = false;
    e = setup_step(machine, UINT64_MAX, cancel, user, &finished);
    if (!e && !finished) e = fail(SF_NOT_FINISHED, "the multigrid setup did not finish");
    if (!e) sys->levels = setup_take_levels(machine);
    setup_destroy(machine);
    if (e) return e;
  } else {
    vector<double> inv(d.n, 1.0);
    for (size_t b = 0; b < rows; ++b) {
      const size_t at = std::lower_bound(sys->cols.begin() + sys->starts[b], sys->cols.begin() + sys->starts[b + 1],
                                         (uint32_t)b) - sys->cols.begin();
      for (int p = 0; p < 3; ++p)
        if (3 * b + p < n) inv[3 * b + p] = 1.0 / bvals[at * 9 + p * 3 + p];
    }
    if ((e = dev_alloc(d, (void**)&d.jacobi, (size_t)d.n * 8))) return e;
    copy_h2d(d, d.jacobi, inv.data(), (size_t)d.n * 8);
  }
  double** vecs[] = {&d.rhs, &d.x, &d.r, &d.z, &d.p, &d.ap};
  for (double** v : vecs)
    if (!e) e = dev_alloc(d, (void**)v, (size_t)d.n * 8);
  if (!e) e = dev_alloc(d, (void**)&d.partials, kReduceBlocks * 4 * 8);
  if (!e) e = dev_alloc(d, (void**)&d.state, sizeof(PcgState));
  if (!e) e = dev_alloc(d, (void**)&d.always_active, sizeof(int));
  if (e) return e;
  vector<double> b(d.n, 0.0);
  std::copy(rhs, rhs + n, b.begin());
  copy_h2d(d, d.rhs, b.data(), (size_t)d.n * 8);
  if (wants_sell(d.system, d.sell_min_rows))
    if ((e = make_sell_from_device(d, d.system, sys->starts.data(), sys->cols.data()))) return e;
  if (mg)
    if ((e = solver_upload_hierarchy(d, sys->levels, o.smoother_degree))) return e;
  if (o.device_memory_budget && d.bytes > o.device_memory_budget)
    return fail(SF_DEVICE_MEMORY_BUDGET, "the system does not fit the device memory budget");
  // PcgOptions::max_iterations defaults to 10 n + 1000 over the caller's unknowns (pcg.rs:138).
  const uint64_t cap = o.max_iterations ? o.max_iterations : 10 * n + 1000;
  e = solver_init_pcg(d, o.tolerance, cap);
  if (!e) e = cuda_check(cudaStreamSynchronize(d.stream), "solver init");
  if (!e && o.use_graphs) e = solver_capture_graph(d);
  if (e) return e;
  sys->pinned = (PcgState*)pinned_slot();
  if (!sys->pinned) return fail(SF_CUDA_ERROR, "cudaMallocHost failed");
  if ((e = solver_read_state(d, &sys->last))) return e;
  sys->status = sys->last.status;
  *out = sys.release();
  return SF_OK;
}

sf_status sf_system_step(sf_system* s, uint64_t max_iterations, sf_cancel_fn cancel, void* user,
                         sf_step_outcome* out) {
  if (!s) return refuse("null argument");
  if (s->cancelled || s->status != ST_ACTIVE) return step_result(s->status, s->cancelled, s->last, out);
  cudaSetDevice(s->solver.device);
  if (sf_status e = run_iterations(s->solver, s->options.use_graphs != 0, max_iterations, cancel, user, s->pinned,
                                   s->last, s->status, s->cancelled))
    return e;
  return step_result(s->status, s->cancelled, s->last, out);
}

sf_status sf_system_estimate(const sf_system* s, double* out) {
  if (!s || !out) return refuse("null argument");
  const DeviceSolver& d = s->solver;
  cudaSetDevice(d.device);
  vector<double> x(d.n);
  copy_d2h(d, x.data(), d.x, (size_t)d.n * 8);
  if (sf_status e = cuda_check(cudaStreamSynchronize(d.stream), "read estimate")) return e;
  std::copy(x.begin(), x.begin() + s->n, out);
  return SF_OK;
}

sf_status sf_system_progress(const sf_system* s, sf_progress* out) {
  if (!s || !out) return refuse("null argument");
  out->iteration = s->last.iterations;
  out->relative_residual = s->last.rel;
  out->at_rounding_floor = s->last.at_floor;
  return SF_OK;
}

uint64_t sf_system_level_count(const sf_system* s) { return s ? s->levels.size() : 0; }

void sf_system_destroy(sf_system* s) {
  if (!s) return;
  cudaSetDevice(s->solver.device);
  delete s;
}

}  // extern "C"
