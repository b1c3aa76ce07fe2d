// The block smoothed-aggregation multigrid setup. It follows the phase sequence of
// crates/solidfem-solve/src/multigrid/setup.rs:242-263 (diagonal, strength, seed, join, sweep,
// group, tentative, spectral, filter, smooth, product, Galerkin, factor) and reproduces the
// reference's aggregates and coarse matrices to the bit.
//
// The split: order-dependent graph work (strong neighbours, the greedy aggregation passes, the
// smoothing filter) and the sparsity patterns P, A P, the coarse matrix and P's transpose are
// built here on the host (the union patterns on the device where they fit); every value of every
// level (inverse diagonal, block norms, lambda_max, the per-aggregate Gram-Schmidt of the
// near-null modes, P, A P, P^T A P) is computed on the device in FP64 (setup_device.cu) and stays
// there. Row-local host work runs on `threads` threads
// in contiguous row chunks stitched back in row order, so the thread count never changes a bit.
// Setup advances in whole phases; the budget counts block rows like the reference's
// (setup.rs:191-222).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <future>
#include <limits>
#include <memory>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "device.h"
#include "sf_internal.h"

namespace sf {

namespace {

const size_t MODES = 6;                 // mod.rs:124
const size_t DENSE_LIMIT = 3000;        // setup.rs:28
const double MAX_COARSE_FRACTION = 0.7; // setup.rs:32
const double RETRY_WIDENING = 1.5;      // setup.rs:36
const size_t MAX_RETRIES = 3;           // setup.rs:37
const int POWER_ITERATIONS = 20;        // setup.rs:41
const double SPECTRAL_MARGIN = 1.15;    // setup.rs:45
const double RANK_TOLERANCE = 1e-10;    // transfer.rs:12

// Splits [0, rows) into `chunks` contiguous ranges and runs f(chunk, begin, end) on each.
template <class F>
void chunked(size_t rows, int threads, F&& f) {
  int chunks = (rows < 4096 || threads <= 1) ? 1 : threads;
#ifdef _OPENMP
#pragma omp parallel for schedule(static, 1) num_threads(chunks) if (chunks > 1)
#endif
  for (int c = 0; c < chunks; ++c) {
    size_t b = rows * (size_t)c / chunks, e = rows * (size_t)(c + 1) / chunks;
    f(c, b, e);
  }
}

template <class F>
void rows_parallel(size_t rows, int threads, F&& f) {
  chunked(rows, threads, [&](int, size_t b, size_t e) {
    for (size_t r = b; r < e; ++r) f(r);
  });
}

// A pattern: per row the sorted distinct columns that `candidates(row, emit)` emits. Columns are
// below `width`; each thread dedupes with its own marker array.
template <class F>
void symbolic_rows(size_t rows, size_t width, int threads, F&& candidates, vector<uint32_t>& starts,
                   vector<uint32_t>& cols) {
  int chunks = (rows < 4096 || threads <= 1) ? 1 : threads;
  vector<vector<uint32_t>> lengths(chunks), parts(chunks);
  chunked(rows, threads, [&](int ci, size_t b, size_t e) {
    vector<uint32_t> mark(width, 0xffffffffu), list;
    vector<uint32_t>& len = lengths[ci];
    vector<uint32_t>& out = parts[ci];
    for (size_t row = b; row < e; ++row) {
      list.clear();
      candidates(row, [&](uint32_t c) {
        if (mark[c] != (uint32_t)row) {
          mark[c] = (uint32_t)row;
          list.push_back(c);
        }
      });
      std::sort(list.begin(), list.end());
      len.push_back((uint32_t)list.size());
      out.insert(out.end(), list.begin(), list.end());
    }
  });
  starts.assign(1, 0);
  starts.reserve(rows + 1);
  size_t total = 0;
  for (auto& p : parts) total += p.size();
  cols.clear();
  cols.reserve(total);
  for (int c = 0; c < chunks; ++c) {
    for (uint32_t l : lengths[c]) starts.push_back(starts.back() + l);
    cols.insert(cols.end(), parts[c].begin(), parts[c].end());
  }
}

double start_value(size_t index) {  // block.rs:379-382
  uint64_t mixed = ((uint64_t)index + 1) * 0x9E3779B97F4A7C15ull;
  return 0.5 + (double)(mixed >> 11) / (double)(1ull << 53);
}

double norm2(const double* x, size_t n) {  // block.rs:398-404, serial in index order
  double s = 0.0;
  for (size_t i = 0; i < n; ++i) s += x[i] * x[i];
  return std::sqrt(s);
}

double squared_distance(const vector<P3>& p, size_t a, size_t b) {
  double dx = p[b][0] - p[a][0], dy = p[b][1] - p[a][1], dz = p[b][2] - p[a][2];
  return dx * dx + dy * dy + dz * dz;
}

// Levels with at least this many block rows find their strong neighbours on the device.
const size_t kDeviceStrengthRows = 16384;

enum Phase { DIAGONAL, STRENGTH, AGGREGATE, TENTATIVE, SPECTRAL, FILTER, SMOOTH, PRODUCT, GALERKIN, FACTOR, DONE };

}  // namespace

struct SetupMachine {
  DeviceSolver& dev;
  SetupOptions opt;
  Phase phase = DIAGONAL;
  Bsr current;  // host pattern, device values
  vector<double> near_null;        // the finest level's modes, on the host until uploaded
  double* d_near_null = nullptr;    // this level's near-null modes on the device, rows x rb x 6
  vector<P3> positions;
  vector<HostLevel> levels;
  // per-level state
  double* inv = nullptr;  // device inverse diagonal
  double* norms = nullptr;  // host copy of the block norms (join pass), a pooled pinned buffer
  bool is_coarsest = false;
  double reach = 3.0;
  size_t retries = 0;
  vector<uint32_t> strong_starts, strong_cols;
  vector<double> closest;
  vector<uint32_t> aggregate;
  size_t aggregates = 0;
  vector<uint32_t> member_starts, members;
  vector<P3> coarse_positions;
  double* d_tentative = nullptr;    // T on the device, rows x rb x 6 (read by the smoothing)
  double* d_coarse_null = nullptr;  // the next level's near-null modes, aggregates x 36
  double lambda_max = 0;
  vector<uint32_t> filter_starts, filter_cols;
  Bsr prolongator, ap, coarse;
  sf_status failure = SF_OK;
  bool cancelled = false;
  // The power iteration needs only the level operator and D^-1, so it runs on a helper thread
  // from the end of the diagonal phase while this thread builds the strength graph and the
  // aggregates (host work that touches neither the device nor these buffers); the tentative phase
  // waits for it before its own device work, the spectral phase takes its result. Declared last,
  // so it is waited for first.
  double *power_v = nullptr, *power_s = nullptr;
  std::future<std::pair<sf_status, double>> power;

  explicit SetupMachine(DeviceSolver& d) : dev(d) {}
  ~SetupMachine() {
    if (power.valid()) power.wait();
    pinned_return(norms);
  }

  size_t level_index() const { return levels.size(); }

  sf_status fail_pd(size_t block, double pivot) {
    error_slot().level = level_index();
    error_slot().block = block;
    error_slot().pivot = pivot;
    return fail(SF_MG_NOT_POSITIVE_DEFINITE, "a multigrid block is not positive definite");
  }

  template <class T>
  sf_status upload(const vector<T>& h, T** d) {
    if (sf_status e = dev_alloc(dev, (void**)d, std::max<size_t>(1, h.size()) * sizeof(T))) return e;
    if (!h.empty()) copy_h2d(dev, *d, h.data(), h.size() * sizeof(T));
    return SF_OK;
  }
  sf_status upload_pattern(Bsr& m) {
    if (sf_status e = upload(m.starts, &m.dev_starts)) return e;
    return upload(m.cols, &m.dev_cols);
  }
  void release(Bsr& m) {
    dev_free(dev, m.dev);
    dev_free(dev, m.dev_starts);
    dev_free(dev, m.dev_cols);
    m = Bsr();
  }
  sf_status sync(const char* what) { return cuda_check(cudaStreamSynchronize(dev.stream), what); }

  // True when a union pattern of `width` columns runs on the device (one warp's bitmap of the
  // columns fits shared memory); wider ones take symbolic_rows on the host.
  static bool union_on_device(size_t width) { return (width + 31) / 32 * 4 <= 200 * 1024; }

  // A union pattern (the symbolic_rows of a product) on the device: a count pass, the row starts
  // by a prefix sum here, a fill pass. `out` gets the device starts and columns and the same
  // arrays on the host, equal to what symbolic_rows gives (each row's distinct columns, sorted).
  sf_status device_union(size_t rows, size_t width, const uint32_t* d_outer_starts, const uint32_t* d_outer_idx,
                         bool self, const uint32_t* d_inner_starts, const uint32_t* d_inner_cols, Bsr& out) {
    sf_status e = dev_alloc(dev, (void**)&out.dev_starts, (rows + 1) * 4);
    if (!e)
      e = setup_union_rows(dev.stream, (uint32_t)rows, (uint32_t)width, d_outer_starts, d_outer_idx, self,
                           d_inner_starts, d_inner_cols, nullptr, out.dev_starts);
    out.starts.assign(rows + 1, 0);
    if (!e && rows) copy_d2h(dev, out.starts.data() + 1, out.dev_starts, rows * 4);
    if (!e) e = sync("union pattern counts");
    if (e) return e;
    for (size_t r = 0; r < rows; ++r) out.starts[r + 1] += out.starts[r];
    copy_h2d(dev, out.dev_starts, out.starts.data(), (rows + 1) * 4);
    const size_t total = out.starts[rows];
    if ((e = dev_alloc(dev, (void**)&out.dev_cols, std::max<size_t>(1, total) * 4))) return e;
    e = setup_union_rows(dev.stream, (uint32_t)rows, (uint32_t)width, d_outer_starts, d_outer_idx, self,
                         d_inner_starts, d_inner_cols, out.dev_starts, out.dev_cols);
    out.cols.resize(total);
    if (!e && total) copy_d2h(dev, out.cols.data(), out.dev_cols, total * 4);
    if (!e) e = sync("union pattern");
    return e;
  }

  // setup.rs:269-321 on the device; the block norms for the join pass come back to the host.
  sf_status run_diagonal() {
    const size_t rb = current.rb, rows = current.rows;
    unsigned long long* bad = nullptr;
    double* pivots = nullptr;
    sf_status e = dev_alloc(dev, (void**)&inv, rows * rb * rb * 8);
    if (!e) e = dev_alloc(dev, (void**)&bad, 8);
    if (!e) e = dev_alloc(dev, (void**)&pivots, std::max<size_t>(1, rows) * 8);
    if (e) return e;
    unsigned long long none = ~0ull;
    copy_h2d(dev, bad, &none, 8);
    e = setup_inverse_diagonal(dev.stream, (uint32_t)rows, (int)rb, current.dev_starts, current.dev_cols, current.dev,
                               inv, bad, pivots);
    unsigned long long first = ~0ull;
    double pivot = 0.0;
    if (!e) {
      copy_d2h(dev, &first, bad, 8);
      e = sync("inverse diagonal");
    }
    if (!e && first != ~0ull) {
      copy_d2h(dev, &pivot, pivots + first, 8);
      e = sync("inverse diagonal");
      if (!e) e = fail_pd((size_t)first, pivot);
    }
    dev_free(dev, bad);
    dev_free(dev, pivots);
    if (e) return e;
    size_t dofs = rows * rb;
    if (dofs <= opt.coarse_dofs || level_index() + 1 >= opt.max_levels) {
      is_coarsest = true;
      phase = SPECTRAL;
      return SF_OK;
    }
    double* d_norms = nullptr;
    size_t blocks = current.cols.size();
    if ((e = dev_alloc(dev, (void**)&d_norms, std::max<size_t>(1, blocks) * 8))) return e;
    e = setup_block_norms(dev.stream, blocks, (int)(rb * current.cb), current.dev, d_norms);
    pinned_return(norms);
    norms = (double*)pinned_acquire(blocks * 8);
    if (!e && !norms) e = fail(SF_CUDA_ERROR, "cudaMallocHost failed");
    if (!e && blocks) copy_d2h(dev, norms, d_norms, blocks * 8);
    if (!e) e = sync("block norms");
    dev_free(dev, d_norms);
    if (!e) e = start_power();
    if (e) return e;
    phase = STRENGTH;
    return SF_OK;
  }

  // Strong neighbours by geometry (aggregate.rs:53-69) on the device for large levels: a count
  // pass with each row's closest distance, the starts summed here, a fill pass; the graph and the
  // distances come back to the host for the aggregation.
  sf_status run_strength_device() {
    const size_t rows = current.rows;
    double *pos = nullptr, *dclosest = nullptr;
    uint32_t *counts = nullptr, *dstarts = nullptr, *dcols = nullptr;
    sf_status e = dev_alloc(dev, (void**)&pos, rows * 24);
    if (!e) e = dev_alloc(dev, (void**)&dclosest, rows * 8);
    if (!e) e = dev_alloc(dev, (void**)&counts, rows * 4);
    if (!e) e = dev_alloc(dev, (void**)&dstarts, (rows + 1) * 4);
    if (!e) {
      copy_h2d(dev, pos, positions.data(), rows * 24);
      e = setup_strength(dev.stream, (uint32_t)rows, current.dev_starts, current.dev_cols, pos, reach * reach, dclosest,
                         nullptr, counts);
    }
    closest.resize(rows);
    strong_starts.assign(rows + 1, 0);
    if (!e) {
      copy_d2h(dev, closest.data(), dclosest, rows * 8);
      copy_d2h(dev, strong_starts.data() + 1, counts, rows * 4);
      e = sync("strength counts");
    }
    if (!e) {
      for (size_t r = 0; r < rows; ++r) strong_starts[r + 1] += strong_starts[r];
      strong_cols.resize(strong_starts[rows]);
      copy_h2d(dev, dstarts, strong_starts.data(), (rows + 1) * 4);
      e = dev_alloc(dev, (void**)&dcols, std::max<size_t>(1, strong_cols.size()) * 4);
    }
    if (!e)
      e = setup_strength(dev.stream, (uint32_t)rows, current.dev_starts, current.dev_cols, pos, reach * reach, nullptr,
                         dstarts, dcols);
    if (!e && !strong_cols.empty()) copy_d2h(dev, strong_cols.data(), dcols, strong_cols.size() * 4);
    if (!e) e = sync("strength");
    for (void* p : {(void*)pos, (void*)dclosest, (void*)counts, (void*)dstarts, (void*)dcols}) dev_free(dev, p);
    if (!e) phase = AGGREGATE;
    return e;
  }

  // Strong neighbours by geometry (aggregate.rs:53-69), two passes so rows run in parallel.
  void run_strength() {
    size_t rows = current.rows;
    closest.assign(rows, 0.0);
    double limit_scale = reach * reach;
    vector<uint32_t> counts(rows, 0);
    // One distance per entry: the row's distances are kept while its closest one is found, and
    // each entry's verdict is marked for the fill pass.
    vector<unsigned char> strong(current.cols.size());
    chunked(rows, opt.threads, [&](int, size_t r0, size_t r1) {
      vector<double> dist;  // this chunk's rows' distances, one row at a time
      const uint32_t* cols = current.cols.data();
      const P3* pos = positions.data();
      for (size_t row = r0; row < r1; ++row) {
        const uint32_t a0 = current.starts[row], a1 = current.starts[row + 1];
        if (dist.size() < a1 - a0) dist.resize(a1 - a0);
        double* d = dist.data();
        double c = std::numeric_limits<double>::max();
        const P3& p = pos[row];
        for (uint32_t at = a0; at < a1; ++at) {
          const uint32_t col = cols[at];
          if (col != row) {
            const P3& q = pos[col];
            const double dx = q[0] - p[0], dy = q[1] - p[1], dz = q[2] - p[2];
            d[at - a0] = dx * dx + dy * dy + dz * dz;  // squared_distance, term for term
            c = std::min(c, d[at - a0]);
          }
        }
        closest[row] = c;
        const double limit = limit_scale * c;
        uint32_t n = 0;
        for (uint32_t at = a0; at < a1; ++at) {
          const bool s = cols[at] != row && d[at - a0] <= limit;
          strong[at] = s;
          n += s;
        }
        counts[row] = n;
      }
    });
    strong_starts.assign(rows + 1, 0);
    for (size_t r = 0; r < rows; ++r) strong_starts[r + 1] = strong_starts[r] + counts[r];
    strong_cols.resize(strong_starts[rows]);
    rows_parallel(rows, opt.threads, [&](size_t row) {
      uint32_t w = strong_starts[row];
      for (uint32_t at = current.starts[row]; at < current.starts[row + 1]; ++at)
        if (strong[at]) strong_cols[w++] = current.cols[at];
    });
    phase = AGGREGATE;
  }

  // Seed, join and sweep passes (aggregate.rs:119-177) then Group (setup_aggregation.rs:165-228).
  void run_aggregate() {
    size_t rows = current.rows;
    aggregate.assign(rows, NO_AGGREGATE);
    vector<char> seeded(rows, 0);
    uint32_t count = 0;
    for (size_t row = 0; row < rows; ++row) {
      uint32_t s = strong_starts[row], e = strong_starts[row + 1];
      if (aggregate[row] != NO_AGGREGATE || s == e) continue;
      bool free_all = true;
      for (uint32_t k = s; k < e && free_all; ++k) free_all = aggregate[strong_cols[k]] == NO_AGGREGATE;
      if (!free_all) continue;
      uint32_t id = count++;
      aggregate[row] = id;
      seeded[row] = 1;
      for (uint32_t k = s; k < e; ++k) {
        aggregate[strong_cols[k]] = id;
        seeded[strong_cols[k]] = 1;
      }
    }
    // join pass: a row's strong neighbours are stamped with the row (the same test as a search
    // of its strong list)
    vector<uint32_t> stamp(rows, NO_AGGREGATE);
    for (size_t row = 0; row < rows; ++row) {
      if (aggregate[row] != NO_AGGREGATE) continue;
      for (uint32_t k = strong_starts[row]; k < strong_starts[row + 1]; ++k) stamp[strong_cols[k]] = (uint32_t)row;
      double best = 0.0;
      uint32_t chosen = NO_AGGREGATE;
      for (uint32_t at = current.starts[row]; at < current.starts[row + 1]; ++at) {
        uint32_t col = current.cols[at];
        if (stamp[col] != (uint32_t)row || !seeded[col]) continue;
        double n = norms[at];
        if (n > best) {
          best = n;
          chosen = aggregate[col];
        }
      }
      if (chosen != NO_AGGREGATE) aggregate[row] = chosen;
    }
    for (size_t row = 0; row < rows; ++row) {
      if (aggregate[row] != NO_AGGREGATE) continue;
      uint32_t id = count++;
      aggregate[row] = id;
      for (uint32_t k = strong_starts[row]; k < strong_starts[row + 1]; ++k)
        if (aggregate[strong_cols[k]] == NO_AGGREGATE) aggregate[strong_cols[k]] = id;
    }
    aggregates = count;
    double coarse_values = (double)(aggregates * MODES);
    bool coarsens = coarse_values <= MAX_COARSE_FRACTION * (double)(rows * current.rb);
    if (!coarsens && retries < MAX_RETRIES) {
      retries += 1;
      reach *= RETRY_WIDENING;
      phase = STRENGTH;
      return;
    }
    if (!coarsens || aggregates == 0) {
      is_coarsest = true;
      aggregates = 0;
      phase = SPECTRAL;
      return;
    }
    member_starts.assign(aggregates + 1, 0);
    for (uint32_t a : aggregate) member_starts[a + 1] += 1;
    for (size_t i = 0; i < aggregates; ++i) member_starts[i + 1] += member_starts[i];
    vector<uint32_t> filled(member_starts.begin(), member_starts.end() - 1);
    members.assign(rows, 0);
    for (size_t row = 0; row < rows; ++row) members[filled[aggregate[row]]++] = (uint32_t)row;
    coarse_positions.assign(aggregates, {0.0, 0.0, 0.0});
    for (size_t a = 0; a < aggregates; ++a) {
      for (uint32_t k = member_starts[a]; k < member_starts[a + 1]; ++k)
        for (int ax = 0; ax < 3; ++ax) coarse_positions[a][ax] += positions[members[k]][ax];
      double cnt = (double)(member_starts[a + 1] - member_starts[a]);
      for (int ax = 0; ax < 3; ++ax) coarse_positions[a][ax] /= cnt;
    }
    phase = TENTATIVE;
  }

  // Tentative prolongator by two-pass Gram-Schmidt per aggregate (transfer.rs:19-68).
  // setup.rs:327-386 on the device (setup_tentative: one thread per aggregate, the host loops'
  // order and bits). The power iteration shares the stream and the solver's counters, so it is
  // waited for first; it started at the end of the diagonal phase and has normally finished while
  // the strength graph and the aggregates were built.
  sf_status run_tentative() {
    const size_t rb = current.rb, rows = current.rows;
    if (power.valid()) power.wait();
    uint32_t *d_starts = nullptr, *d_members = nullptr;
    sf_status e = SF_OK;
    if (!d_near_null) {  // the finest level's modes come from the host
      e = upload(near_null, &d_near_null);
      vector<double>().swap(near_null);
    }
    if (!e) e = upload(member_starts, &d_starts);
    if (!e) e = upload(members, &d_members);
    if (!e) e = dev_alloc(dev, (void**)&d_tentative, std::max<size_t>(1, rows * rb * MODES) * 8);
    if (!e) e = dev_alloc(dev, (void**)&d_coarse_null, std::max<size_t>(1, aggregates) * 36 * 8);
    size_t max_members = 0;
    for (size_t a = 0; a < aggregates; ++a) max_members = std::max<size_t>(max_members, member_starts[a + 1] - member_starts[a]);
    if (!e)
      e = setup_tentative(dev.stream, aggregates, (int)rb, max_members, d_starts, d_members, d_near_null, d_tentative,
                          d_coarse_null);
    // stream-ordered frees: after the kernel that reads them
    for (void* p : {(void*)d_starts, (void*)d_members, (void*)d_near_null}) dev_free(dev, p);
    d_near_null = nullptr;
    if (e) return e;
    phase = SPECTRAL;
    return SF_OK;
  }

  // Power iteration for lambda_max(D^-1 A) (setup.rs:390-449): the products on the device, the
  // order-exact norms on the host from a pinned copy of each iterate. Returns the last norm.
  std::pair<sf_status, double> power_iteration() {
    cudaSetDevice(dev.device);  // a helper thread starts on device 0
    const size_t rb = current.rb, rows = current.rows, dofs = rows * rb;
    double* pinned = (double*)pinned_acquire(std::max<size_t>(1, dofs) * 8);
    if (!pinned) return {SF_CUDA_ERROR, 0.0};
    sf_status e = SF_OK;
    double lm = 0.0;
    if (dofs) {
      double* v = power_v;
      double* s2 = power_s;
      for (size_t i = 0; i < dofs; ++i) pinned[i] = start_value(i);
      double n0 = norm2(pinned, dofs);
      for (size_t i = 0; i < dofs; ++i) pinned[i] /= n0;
      copy_h2d(dev, v, pinned, dofs * 8);
      // Each iterate comes back in chunks, each with an event: the host's serial sum of squares
      // (norm2's order) starts on the first chunk while the rest are still in flight.
      constexpr int kChunks = 8;
      cudaEvent_t landed[kChunks];
      for (int c = 0; c < kChunks; ++c) cudaEventCreateWithFlags(&landed[c], cudaEventDisableTiming);
      const size_t chunk = (dofs + kChunks - 1) / kChunks;
      for (int it = 0; it < POWER_ITERATIONS && !e; ++it) {
        e = setup_power_step(dev.stream, (uint32_t)rows, (int)rb, current.dev_starts, current.dev_cols, current.dev,
                             inv, v, s2);
        for (int c = 0; c < kChunks && !e; ++c) {
          const size_t at = std::min(dofs, c * chunk), len = std::min(dofs, at + chunk) - at;
          if (len) copy_d2h(dev, pinned + at, s2 + at, len * 8);
          cudaEventRecord(landed[c], dev.stream);
        }
        double sum = 0.0;
        for (int c = 0; c < kChunks && !e; ++c) {
          e = cuda_check(cudaEventSynchronize(landed[c]), "power iteration");
          const size_t at = std::min(dofs, c * chunk), end = std::min(dofs, at + chunk);
          for (size_t i = at; i < end; ++i) sum += pinned[i] * pinned[i];
        }
        if (!e) {
          double n = std::sqrt(sum);  // norm2 (block.rs:398-404), the same serial sum
          lm = n;
          e = setup_scale(dev.stream, dofs, s2, n, v);
        }
      }
      if (!e) e = sync("power iteration");
      else cudaStreamSynchronize(dev.stream);
      for (int c = 0; c < kChunks; ++c) cudaEventDestroy(landed[c]);
    }
    pinned_return(pinned);  // every copy from it completed at the syncs
    return {e, lm};
  }

  sf_status start_power() {
    const size_t dofs = current.rows * current.rb;
    sf_status e = dev_alloc(dev, (void**)&power_v, std::max<size_t>(1, dofs) * 8);
    if (!e) e = dev_alloc(dev, (void**)&power_s, std::max<size_t>(1, dofs) * 8);
    if (e) return e;
    power = std::async(std::launch::async, [this] { return power_iteration(); });
    return SF_OK;
  }

  sf_status run_spectral() {
    const size_t rb = current.rb, rows = current.rows;
    if (!power.valid())
      if (sf_status e = start_power()) return e;
    std::pair<sf_status, double> r = power.get();
    dev_free(dev, power_v);
    dev_free(dev, power_s);
    power_v = power_s = nullptr;
    if (r.first) return fail(r.first, "the power iteration for the largest eigenvalue failed");
    lambda_max = r.second * SPECTRAL_MARGIN;
    if (is_coarsest) {
      phase = (rows * rb <= DENSE_LIMIT) ? FACTOR : DONE;
      if (phase == DONE) push_final(false);
      return SF_OK;
    }
    phase = FILTER;
    return SF_OK;
  }

  // Smoothing neighbours of a coarse level (aggregate.rs:80-96); the finest keeps its strong ones.
  void run_filter() {
    filter_starts.clear();
    filter_cols.clear();
    if (level_index() > 0) {
      size_t rows = current.rows;
      double rr = reach * reach;
      vector<uint32_t> counts(rows, 0);
      vector<double> limits(rows, 0.0);
      rows_parallel(rows, opt.threads, [&](size_t row) {
        double scale = closest[row];
        for (uint32_t at = current.starts[row]; at < current.starts[row + 1]; ++at) {
          uint32_t c = current.cols[at];
          if (c != row) scale = std::max(scale, closest[c]);
        }
        double limit = rr * scale;
        limits[row] = limit;
        uint32_t n = 0;
        for (uint32_t at = current.starts[row]; at < current.starts[row + 1]; ++at) {
          uint32_t c = current.cols[at];
          if (c != row && squared_distance(positions, row, c) <= limit) ++n;
        }
        counts[row] = n;
      });
      filter_starts.assign(rows + 1, 0);
      for (size_t r = 0; r < rows; ++r) filter_starts[r + 1] = filter_starts[r] + counts[r];
      filter_cols.assign(filter_starts[rows], 0);
      rows_parallel(rows, opt.threads, [&](size_t row) {
        uint32_t w = filter_starts[row];
        for (uint32_t at = current.starts[row]; at < current.starts[row + 1]; ++at) {
          uint32_t c = current.cols[at];
          if (c != row && squared_distance(positions, row, c) <= limits[row]) filter_cols[w++] = c;
        }
      });
    }
    phase = SMOOTH;
  }

  // The row of every entry of a pattern, on the device.
  sf_status entry_rows(const Bsr& m, uint32_t** out) {
    if (sf_status e = dev_alloc(dev, (void**)out, std::max<size_t>(1, m.cols.size()) * 4)) return e;
    return setup_entry_rows(dev.stream, (uint32_t)m.rows, m.dev_starts, *out);
  }

  // P = T - omega D^-1 A_f T (transfer.rs:108-152). P's pattern: the row's own aggregate and the
  // aggregates of its smoothing neighbours; its values on the device.
  sf_status run_smooth() {
    double omega = 4.0 / (3.0 * lambda_max);
    size_t rb = current.rb, rows = current.rows;
    const vector<uint32_t>& ns = filter_starts.empty() ? strong_starts : filter_starts;
    const vector<uint32_t>& nc = filter_starts.empty() ? strong_cols : filter_cols;
    prolongator = Bsr();
    prolongator.rows = rows;
    prolongator.rb = rb;
    prolongator.cb = MODES;
    uint32_t *n_starts = nullptr, *n_cols = nullptr, *agg = nullptr, *rows_of = nullptr;
    sf_status e = upload(ns, &n_starts);
    if (!e) e = upload(nc, &n_cols);
    if (!e) e = upload(aggregate, &agg);
    if (!e && union_on_device(aggregates)) {
      // the row's own aggregate and its neighbours' aggregates
      e = device_union(rows, aggregates, n_starts, n_cols, true, nullptr, agg, prolongator);
    } else if (!e) {
      symbolic_rows(
          rows, aggregates, opt.threads,
          [&](size_t row, auto&& emit) {
            emit(aggregate[row]);
            for (uint32_t k = ns[row]; k < ns[row + 1]; ++k) emit(aggregate[nc[k]]);
          },
          prolongator.starts, prolongator.cols);
      e = upload_pattern(prolongator);
    }
    size_t entries = prolongator.cols.size();
    double* t = d_tentative;
    d_tentative = nullptr;
    if (!e) e = dev_alloc(dev, (void**)&prolongator.dev, std::max<size_t>(1, entries) * rb * MODES * 8);
    if (!e) e = entry_rows(prolongator, &rows_of);
    if (!e)
      e = setup_smooth(dev.stream, (int)rb, entries, rows_of, prolongator.dev_cols, current.dev_starts,
                       current.dev_cols, current.dev, n_starts, n_cols, agg, t, inv, omega, prolongator.dev);
    if (!e) e = sync("smooth");
    for (void* p : {(void*)n_starts, (void*)n_cols, (void*)agg, (void*)rows_of, (void*)t}) dev_free(dev, p);
    if (e) return e;
    phase = PRODUCT;
    return SF_OK;
  }

  // A P (transfer.rs:155-169): pattern the union of P's rows at A's columns.
  sf_status run_product() {
    size_t rb = current.rb, rows = current.rows;
    ap = Bsr();
    ap.rows = rows;
    ap.rb = rb;
    ap.cb = MODES;
    sf_status e = SF_OK;
    if (union_on_device(aggregates)) {
      e = device_union(rows, aggregates, current.dev_starts, current.dev_cols, false, prolongator.dev_starts,
                       prolongator.dev_cols, ap);
    } else {
      symbolic_rows(
          rows, aggregates, opt.threads,
          [&](size_t row, auto&& emit) {
            for (uint32_t at = current.starts[row]; at < current.starts[row + 1]; ++at) {
              uint32_t col = current.cols[at];
              for (uint32_t in = prolongator.starts[col]; in < prolongator.starts[col + 1]; ++in)
                emit(prolongator.cols[in]);
            }
          },
          ap.starts, ap.cols);
      e = upload_pattern(ap);
    }
    uint32_t* rows_of = nullptr;
    size_t entries = ap.cols.size();
    if (!e) e = dev_alloc(dev, (void**)&ap.dev, std::max<size_t>(1, entries) * rb * MODES * 8);
    if (!e) e = entry_rows(ap, &rows_of);
    if (!e)
      e = setup_product(dev.stream, (int)rb, entries, rows_of, ap.dev_cols, current.dev_starts, current.dev_cols,
                        current.dev, prolongator.dev_starts, prolongator.dev_cols, prolongator.dev, ap.dev);
    if (!e) e = sync("product");
    dev_free(dev, rows_of);
    if (e) return e;
    phase = GALERKIN;
    return SF_OK;
  }

  // P^T (A P) by coarse row, P read by columns with fine rows ascending (transfer.rs:173-238).
  sf_status run_galerkin() {
    const size_t cdim = MODES;
    vector<uint32_t> pt_starts(aggregates + 1, 0);
    for (uint32_t c : prolongator.cols) pt_starts[c + 1] += 1;
    for (size_t i = 0; i < aggregates; ++i) pt_starts[i + 1] += pt_starts[i];
    vector<uint32_t> filled(pt_starts.begin(), pt_starts.end() - 1);
    vector<uint32_t> pt_rows(prolongator.cols.size()), pt_at(prolongator.cols.size());
    for (size_t row = 0; row < prolongator.rows; ++row)
      for (uint32_t at = prolongator.starts[row]; at < prolongator.starts[row + 1]; ++at) {
        uint32_t o = filled[prolongator.cols[at]]++;
        pt_rows[o] = (uint32_t)row;
        pt_at[o] = at;
      }
    coarse = Bsr();
    coarse.rows = aggregates;
    coarse.rb = coarse.cb = cdim;
    uint32_t *d_pt_starts = nullptr, *d_pt_rows = nullptr, *d_pt_at = nullptr, *rows_of = nullptr;
    sf_status e = upload(pt_starts, &d_pt_starts);
    if (!e) e = upload(pt_rows, &d_pt_rows);
    if (!e) e = upload(pt_at, &d_pt_at);
    if (!e && union_on_device(aggregates)) {
      e = device_union(aggregates, aggregates, d_pt_starts, d_pt_rows, false, ap.dev_starts, ap.dev_cols, coarse);
    } else if (!e) {
      symbolic_rows(
          aggregates, aggregates, opt.threads,
          [&](size_t c, auto&& emit) {
            for (uint32_t k = pt_starts[c]; k < pt_starts[c + 1]; ++k) {
              uint32_t fine_row = pt_rows[k];
              for (uint32_t in = ap.starts[fine_row]; in < ap.starts[fine_row + 1]; ++in) emit(ap.cols[in]);
            }
          },
          coarse.starts, coarse.cols);
      e = upload_pattern(coarse);
    }
    size_t entries = coarse.cols.size();
    if (!e) e = dev_alloc(dev, (void**)&coarse.dev, std::max<size_t>(1, entries) * cdim * cdim * 8);
    if (!e) e = entry_rows(coarse, &rows_of);
    if (!e)
      e = setup_galerkin(dev.stream, (int)prolongator.rb, entries, rows_of, coarse.dev_cols, d_pt_starts, d_pt_rows,
                         d_pt_at, prolongator.dev, ap.dev_starts, ap.dev_cols, ap.dev, coarse.dev);
    if (!e) e = sync("galerkin");
    for (void* p : {(void*)d_pt_starts, (void*)d_pt_rows, (void*)d_pt_at, (void*)rows_of}) dev_free(dev, p);
    release(ap);
    if (e) return e;
    HostLevel lv;
    lv.a = std::move(current);
    lv.inverse_diagonal = inv;
    inv = nullptr;
    lv.lambda_max = lambda_max;
    lv.lambda_min = lambda_max / opt.range;
    lv.has_p = true;
    lv.p = std::move(prolongator);
    lv.aggregates = std::move(aggregate);
    levels.push_back(std::move(lv));
    current = std::move(coarse);
    coarse = Bsr();
    prolongator = Bsr();
    d_near_null = d_coarse_null;
    d_coarse_null = nullptr;
    positions = std::move(coarse_positions);
    pinned_return(norms);
    norms = nullptr;
    reach = opt.reach;
    retries = 0;
    is_coarsest = false;
    aggregates = 0;
    phase = DIAGONAL;
    return SF_OK;
  }

  void push_final(bool factored) {
    dev_free(dev, d_near_null);  // the coarsest level's modes are not needed
    d_near_null = nullptr;
    HostLevel lv;
    lv.a = std::move(current);
    lv.inverse_diagonal = inv;
    inv = nullptr;
    lv.lambda_max = lambda_max;
    lv.lambda_min = lambda_max / opt.range;
    lv.has_factor = factored;
    levels.push_back(std::move(lv));
  }

  // Dense Cholesky of the coarsest level (block.rs:307-374), then its explicit inverse
  // L^-T L^-1, which the device applies as one matrix-vector product per cycle: both on the device
  // in FP64 (setup_dense_inverse, the host loops' bits); the first non-positive pivot is refused.
  sf_status run_factor() {
    const size_t n = current.rows * current.rb, nn = std::max<size_t>(1, n * n) * 8;
    double *work = nullptr, *li = nullptr, *inverse = nullptr, *pivot = nullptr;
    unsigned long long* bad = nullptr;
    sf_status e = dev_alloc(dev, (void**)&work, nn);
    if (!e) e = dev_alloc(dev, (void**)&li, nn);
    if (!e) e = dev_alloc(dev, (void**)&inverse, nn);
    if (!e) e = dev_alloc(dev, (void**)&bad, 8);
    if (!e) e = dev_alloc(dev, (void**)&pivot, 8);
    unsigned long long first = ~0ull;
    double value = 0.0;
    if (!e) {
      copy_h2d(dev, bad, &first, 8);
      e = setup_dense_inverse(dev.stream, (uint32_t)current.rows, (int)current.rb, current.dev_starts, current.dev_cols,
                              current.dev, n, work, li, inverse, bad, pivot);
    }
    if (!e) {
      copy_d2h(dev, &first, bad, 8);
      copy_d2h(dev, &value, pivot, 8);
      e = sync("coarsest factor");
    }
    for (void* p : {(void*)work, (void*)li, (void*)bad, (void*)pivot}) dev_free(dev, p);
    if (!e && first != ~0ull) e = fail_pd((size_t)first, value);
    if (e) {
      dev_free(dev, inverse);
      return e;
    }
    HostLevel lv;
    lv.dev_coarse_inverse = inverse;
    lv.factor_n = n;
    lv.a = std::move(current);
    lv.inverse_diagonal = inv;
    inv = nullptr;
    lv.lambda_max = lambda_max;
    lv.lambda_min = lambda_max / opt.range;
    lv.has_factor = true;
    levels.push_back(std::move(lv));
    phase = DONE;
    return SF_OK;
  }
};

SetupMachine* setup_create(DeviceSolver& solver, Bsr&& fine, vector<double>&& near_null, vector<P3>&& positions,
                           const SetupOptions& options, double* device_near_null) {
  SetupMachine* m = new SetupMachine(solver);
  m->opt = options;
  m->current = std::move(fine);
  m->near_null = std::move(near_null);
  m->d_near_null = device_near_null;
  m->positions = std::move(positions);
  m->reach = options.reach;
  return m;
}

sf_status setup_step(SetupMachine* m, size_t budget, sf_cancel_fn cancel, void* user, bool* finished) {
  if (m->failure) return fail(m->failure, "the multigrid setup failed earlier");
  if (m->cancelled) return fail(SF_CANCELLED, "the multigrid setup was cancelled");
  size_t spent = 0;
  while (m->phase != DONE) {
    if (spent >= budget) break;
    if (cancel && cancel(user)) {
      m->cancelled = true;
      return fail(SF_CANCELLED, "the multigrid setup was cancelled");
    }
    size_t rows = m->current.rows;
    sf_status s = SF_OK;
    switch (m->phase) {
      case DIAGONAL: s = m->run_diagonal(); break;
      case STRENGTH:
        if (m->current.rows >= kDeviceStrengthRows && m->current.dev_starts && m->current.dev_cols)
          s = m->run_strength_device();
        else
          m->run_strength();
        break;
      case AGGREGATE: m->run_aggregate(); break;
      case TENTATIVE: s = m->run_tentative(); break;
      case SPECTRAL:
        s = m->run_spectral();
        rows *= 20;
        break;
      case FILTER: m->run_filter(); break;
      case SMOOTH: s = m->run_smooth(); break;
      case PRODUCT: s = m->run_product(); break;
      case GALERKIN: s = m->run_galerkin(); break;
      case FACTOR: s = m->run_factor(); break;
      case DONE: break;
    }
    if (s != SF_OK) {
      m->failure = s;
      return s;
    }
    spent += std::max<size_t>(rows, 1);
  }
  *finished = m->phase == DONE;
  return SF_OK;
}

vector<HostLevel> setup_take_levels(SetupMachine* m) { return std::move(m->levels); }
void setup_destroy(SetupMachine* m) { delete m; }

}  // namespace sf
