// The block smoothed-aggregation multigrid setup, host side. It follows the phase sequence of
// crates/solidfem-solve/src/multigrid/setup.rs:242-263 (diagonal, strength, seed, join, sweep,
// group, tentative, spectral, filter, smooth, product, Galerkin, factor) with every floating-point
// operation in the reference's order, so the aggregates and every coarse matrix are the
// reference's to the bit. The aggregation passes are order-dependent graph work and run serially;
// every row-local phase runs on `threads` host threads in contiguous row chunks that are stitched
// back in row order, so the thread count never changes a bit. Setup advances in whole phases; the
// budget counts block rows like the reference's (setup.rs:191-222).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <limits>
#include <memory>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "sf_internal.h"

namespace sf {

namespace {

const size_t MODES = 6;                 // mod.rs:124
const size_t DENSE_LIMIT = 3000;        // setup.rs:28
const double MAX_COARSE_FRACTION = 0.7; // setup.rs:32
const double RETRY_WIDENING = 1.5;      // setup.rs:36
const size_t MAX_RETRIES = 3;           // setup.rs:37
const size_t POWER_ITERATIONS = 20;     // setup.rs:41
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

// C += A B for row-major dense blocks (block.rs:229-245), same loop order.
inline void add_product(double* out, const double* a, size_t a_rows, size_t middle, const double* b, size_t b_cols) {
  for (size_t r = 0; r < a_rows; ++r)
    for (size_t m = 0; m < middle; ++m) {
      double s = a[r * middle + m];
      for (size_t c = 0; c < b_cols; ++c) out[r * b_cols + c] += s * b[m * b_cols + c];
    }
}

// Cholesky-based SPD block inverse (block.rs:186-224).
bool invert_spd_block(const double* in, size_t n, double* out, double* pivot) {
  double lower[36] = {0};
  for (size_t i = 0; i < n; ++i)
    for (size_t j = 0; j <= i; ++j) {
      double sum = in[i * n + j];
      for (size_t k = 0; k < j; ++k) sum -= lower[i * n + k] * lower[j * n + k];
      if (i == j) {
        if (!std::isfinite(sum) || sum <= 0.0) {
          *pivot = sum;
          return false;
        }
        lower[i * n + j] = std::sqrt(sum);
      } else {
        lower[i * n + j] = sum / lower[j * n + j];
      }
    }
  double inv[36] = {0};
  for (size_t c = 0; c < n; ++c)
    for (size_t i = c; i < n; ++i) {
      double sum = i == c ? 1.0 : 0.0;
      for (size_t k = c; k < i; ++k) sum -= lower[i * n + k] * inv[k * n + c];
      inv[i * n + c] = sum / lower[i * n + i];
    }
  for (size_t i = 0; i < n; ++i)
    for (size_t j = 0; j < n; ++j) {
      double sum = 0.0;
      for (size_t k = std::max(i, j); k < n; ++k) sum += inv[k * n + i] * inv[k * n + j];
      out[i * n + j] = sum;
    }
  return true;
}

// A sparse row whose block columns arrive in any order, read back sorted (block.rs:249-302).
struct RowAccumulator {
  vector<uint32_t> slot, touched;
  vector<double> data;
  size_t len;
  RowAccumulator(size_t columns, size_t block_len) : slot(columns, 0xffffffffu), len(block_len) {}
  void begin() {
    for (uint32_t c : touched) slot[c] = 0xffffffffu;
    touched.clear();
    data.clear();
  }
  double* entry(uint32_t c) {
    uint32_t at = slot[c];
    if (at == 0xffffffffu) {
      at = (uint32_t)touched.size();
      slot[c] = at;
      touched.push_back(c);
      data.resize(data.size() + len, 0.0);
    }
    return data.data() + (size_t)at * len;
  }
  template <class F>
  void drain(F&& emit) {
    std::sort(touched.begin(), touched.end());
    for (uint32_t c : touched) emit(c, data.data() + (size_t)slot[c] * len);
  }
};

// A chunk of consecutive output rows built by one thread.
struct RowChunk {
  vector<uint32_t> lengths, cols;
  vector<double> vals;
};

void stitch(vector<RowChunk>& chunks, size_t rows, size_t rb, size_t cb, Bsr& out) {
  out.rows = rows;
  out.rb = rb;
  out.cb = cb;
  size_t total = 0;
  for (auto& c : chunks) total += c.cols.size();
  out.starts.assign(1, 0);
  out.starts.reserve(rows + 1);
  out.cols.clear();
  out.cols.reserve(total);
  out.vals.clear();
  out.vals.reserve(total * rb * cb);
  for (auto& c : chunks) {
    for (uint32_t l : c.lengths) out.starts.push_back(out.starts.back() + l);
    out.cols.insert(out.cols.end(), c.cols.begin(), c.cols.end());
    out.vals.insert(out.vals.end(), c.vals.begin(), c.vals.end());
    c = RowChunk();
  }
}

double squared_distance(const vector<P3>& p, size_t a, size_t b) {
  double dx = p[b][0] - p[a][0], dy = p[b][1] - p[a][1], dz = p[b][2] - p[a][2];
  return dx * dx + dy * dy + dz * dz;
}

double block_norm(const double* b, size_t len) {
  double s = 0.0;
  for (size_t i = 0; i < len; ++i) s += b[i] * b[i];
  return std::sqrt(s);
}

double start_value(size_t index) {  // block.rs:379-382
  uint64_t mixed = ((uint64_t)index + 1) * 0x9E3779B97F4A7C15ull;
  return 0.5 + (double)(mixed >> 11) / (double)(1ull << 53);
}

double norm2(const vector<double>& x) {  // block.rs:398-404, serial in index order
  double s = 0.0;
  for (double v : x) s += v * v;
  return std::sqrt(s);
}

enum Phase { DIAGONAL, STRENGTH, AGGREGATE, TENTATIVE, SPECTRAL, FILTER, SMOOTH, PRODUCT, GALERKIN, FACTOR, DONE };

}  // namespace

struct SetupMachine {
  SetupOptions opt;
  Phase phase = DIAGONAL;
  Bsr current;
  vector<double> near_null;
  vector<P3> positions;
  vector<HostLevel> levels;
  // per-level state
  vector<double> inv;
  bool is_coarsest = false;
  double reach = 3.0;
  size_t retries = 0;
  vector<uint32_t> strong_starts, strong_cols;
  vector<double> closest;
  vector<uint32_t> aggregate;
  size_t aggregates = 0;
  vector<uint32_t> member_starts, members;
  vector<P3> coarse_positions;
  Bsr tentative;
  vector<double> coarse_null;
  double lambda_max = 0;
  vector<uint32_t> filter_starts, filter_cols;
  Bsr prolongator, ap, coarse;
  sf_status failure = SF_OK;
  bool cancelled = false;

  size_t level_index() const { return levels.size(); }

  sf_status fail_pd(size_t block, double pivot) {
    error_slot().level = level_index();
    error_slot().block = block;
    error_slot().pivot = pivot;
    return fail(SF_MG_NOT_POSITIVE_DEFINITE, "a multigrid block is not positive definite");
  }

  // setup.rs:269-321
  sf_status run_diagonal() {
    size_t rb = current.rb;
    inv.assign(current.rows * rb * rb, 0.0);
    std::atomic_size_t bad(SIZE_MAX);
    vector<double> pivots(current.rows, 0.0);
    rows_parallel(current.rows, opt.threads, [&](size_t row) {
      const uint32_t* b = current.cols.data() + current.starts[row];
      const uint32_t* e = current.cols.data() + current.starts[row + 1];
      const uint32_t* it = std::lower_bound(b, e, (uint32_t)row);
      double pivot = 0.0;
      bool ok = it != e && *it == row &&
                invert_spd_block(current.block(it - current.cols.data()), rb, inv.data() + row * rb * rb, &pivot);
      if (!ok) {
        pivots[row] = pivot;
        size_t prev = bad.load();
        while (row < prev && !bad.compare_exchange_weak(prev, row)) {
        }
      }
    });
    if (bad.load() != SIZE_MAX) return fail_pd(bad.load(), pivots[bad.load()]);
    size_t dofs = current.rows * rb;
    if (dofs <= opt.coarse_dofs || level_index() + 1 >= opt.max_levels) {
      is_coarsest = true;
      phase = SPECTRAL;
    } else {
      phase = STRENGTH;
    }
    return SF_OK;
  }

  // Strong neighbours by geometry (aggregate.rs:53-69), two passes so rows run in parallel.
  void run_strength() {
    size_t rows = current.rows;
    closest.assign(rows, 0.0);
    double limit_scale = reach * reach;
    vector<uint32_t> counts(rows, 0);
    rows_parallel(rows, opt.threads, [&](size_t row) {
      double c = std::numeric_limits<double>::max();
      for (uint32_t at = current.starts[row]; at < current.starts[row + 1]; ++at) {
        uint32_t col = current.cols[at];
        if (col != row) c = std::min(c, squared_distance(positions, row, col));
      }
      closest[row] = c;
      double limit = limit_scale * c;
      uint32_t n = 0;
      for (uint32_t at = current.starts[row]; at < current.starts[row + 1]; ++at) {
        uint32_t col = current.cols[at];
        if (col != row && squared_distance(positions, row, col) <= limit) ++n;
      }
      counts[row] = n;
    });
    strong_starts.assign(rows + 1, 0);
    for (size_t r = 0; r < rows; ++r) strong_starts[r + 1] = strong_starts[r] + counts[r];
    strong_cols.assign(strong_starts[rows], 0);
    rows_parallel(rows, opt.threads, [&](size_t row) {
      double limit = limit_scale * closest[row];
      uint32_t w = strong_starts[row];
      for (uint32_t at = current.starts[row]; at < current.starts[row + 1]; ++at) {
        uint32_t col = current.cols[at];
        if (col != row && squared_distance(positions, row, col) <= limit) strong_cols[w++] = col;
      }
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
    size_t bl = current.rb * current.cb;
    for (size_t row = 0; row < rows; ++row) {
      if (aggregate[row] != NO_AGGREGATE) continue;
      const uint32_t* nb = strong_cols.data() + strong_starts[row];
      const uint32_t* ne = strong_cols.data() + strong_starts[row + 1];
      double best = 0.0;
      uint32_t chosen = NO_AGGREGATE;
      for (uint32_t at = current.starts[row]; at < current.starts[row + 1]; ++at) {
        uint32_t col = current.cols[at];
        if (!std::binary_search(nb, ne, col) || !seeded[col]) continue;
        double n = block_norm(current.block(at), bl);
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
  void run_tentative() {
    size_t rb = current.rb, rows = current.rows, block = rb * MODES;
    tentative.rows = rows;
    tentative.rb = rb;
    tentative.cb = MODES;
    tentative.starts.resize(rows + 1);
    for (size_t r = 0; r <= rows; ++r) tentative.starts[r] = (uint32_t)r;
    tentative.cols = aggregate;
    tentative.vals.assign(rows * block, 0.0);
    coarse_null.assign(aggregates * 36, 0.0);
    rows_parallel(aggregates, opt.threads, [&](size_t a) {
      size_t count = member_starts[a + 1] - member_starts[a];
      const uint32_t* mem = members.data() + member_starts[a];
      size_t lrows = count * rb;
      vector<double> local(lrows * MODES);
      for (size_t m = 0; m < count; ++m)
        for (size_t p = 0; p < rb; ++p)
          for (size_t k = 0; k < MODES; ++k)
            local[(m * rb + p) * MODES + k] = near_null[((size_t)mem[m] * rb + p) * MODES + k];
      double* coarse = coarse_null.data() + a * 36;
      auto column_norm = [&](size_t c) {
        double s = 0.0;
        for (size_t r = 0; r < lrows; ++r) s += local[r * MODES + c] * local[r * MODES + c];
        return std::sqrt(s);
      };
      for (size_t c = 0; c < MODES; ++c) {
        double original = column_norm(c);
        for (int pass = 0; pass < 2; ++pass)
          for (size_t prev = 0; prev < c; ++prev) {
            double proj = 0.0;
            for (size_t r = 0; r < lrows; ++r) proj += local[r * MODES + prev] * local[r * MODES + c];
            coarse[prev * MODES + c] += proj;
            for (size_t r = 0; r < lrows; ++r) local[r * MODES + c] -= proj * local[r * MODES + prev];
          }
        double rem = column_norm(c);
        if (original == 0.0 || rem <= RANK_TOLERANCE * original) {
          for (size_t r = 0; r < lrows; ++r) local[r * MODES + c] = 0.0;
          coarse[c * MODES + c] = 0.0;
        } else {
          for (size_t r = 0; r < lrows; ++r) local[r * MODES + c] /= rem;
          coarse[c * MODES + c] = rem;
        }
      }
      for (size_t m = 0; m < count; ++m)
        std::copy(local.begin() + m * block, local.begin() + (m + 1) * block,
                  tentative.vals.begin() + (size_t)mem[m] * block);
    });
    phase = SPECTRAL;
  }

  // Power iteration for lambda_max(D^-1 A) (setup.rs:390-449): row-parallel products, serial norm.
  void run_spectral() {
    size_t rb = current.rb, rows = current.rows, dofs = rows * rb;
    vector<double> v(dofs), s2(dofs);
    for (size_t i = 0; i < dofs; ++i) v[i] = start_value(i);
    double n0 = norm2(v);
    for (double& x : v) x /= n0;
    double lm = 0.0;
    for (size_t it = 0; it < POWER_ITERATIONS; ++it) {
      rows_parallel(rows, opt.threads, [&](size_t row) {
        double y[6] = {0, 0, 0, 0, 0, 0};
        for (uint32_t at = current.starts[row]; at < current.starts[row + 1]; ++at) {
          const double* b = current.block(at);
          size_t col = (size_t)current.cols[at] * current.cb;
          for (size_t p = 0; p < rb; ++p) {
            double sum = y[p];
            for (size_t q = 0; q < current.cb; ++q) sum += b[p * current.cb + q] * v[col + q];
            y[p] = sum;
          }
        }
        const double* d = inv.data() + row * rb * rb;
        for (size_t p = 0; p < rb; ++p) {
          double sum = 0.0;
          for (size_t q = 0; q < rb; ++q) sum += d[p * rb + q] * y[q];
          s2[row * rb + p] = sum;
        }
      });
      double n = norm2(s2);
      lm = n;
      rows_parallel(dofs, opt.threads, [&](size_t i) { v[i] = s2[i] / n; });
    }
    lambda_max = lm * SPECTRAL_MARGIN;
    if (is_coarsest) {
      phase = (rows * rb <= DENSE_LIMIT) ? FACTOR : DONE;
      if (phase == DONE) push_final(false);
      return;
    }
    phase = FILTER;
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

  // P = T - omega D^-1 A_f T, row by row (transfer.rs:108-152).
  void run_smooth() {
    double omega = 4.0 / (3.0 * lambda_max);
    size_t rb = current.rb, cb = MODES, rows = current.rows;
    int chunks = (rows < 4096 || opt.threads <= 1) ? 1 : opt.threads;
    vector<RowChunk> out(chunks);
    const vector<uint32_t>& ns = filter_starts.empty() ? strong_starts : filter_starts;
    const vector<uint32_t>& nc = filter_starts.empty() ? strong_cols : filter_cols;
    chunked(rows, opt.threads, [&](int ci, size_t b, size_t e) {
      RowAccumulator acc(aggregates, rb * cb);
      RowChunk& o = out[ci];
      vector<double> scaled(rb * cb);
      for (size_t row = b; row < e; ++row) {
        acc.begin();
        uint32_t t_col = tentative.cols[row];
        acc.entry(t_col);
        const uint32_t* nb = nc.data() + ns[row];
        const uint32_t* ne = nc.data() + ns[row + 1];
        for (uint32_t at = current.starts[row]; at < current.starts[row + 1]; ++at) {
          uint32_t col = current.cols[at];
          size_t src = (col == row || std::binary_search(nb, ne, col)) ? col : row;
          double* acc_block = acc.entry(tentative.cols[src]);
          add_product(acc_block, current.block(at), rb, current.cb, tentative.block(src), cb);
        }
        const double* dinv = inv.data() + row * rb * rb;
        const double* t_block = tentative.block(row);
        uint32_t n = 0;
        acc.drain([&](uint32_t col, const double* blk) {
          std::fill(scaled.begin(), scaled.end(), 0.0);
          add_product(scaled.data(), dinv, rb, rb, blk, cb);
          o.cols.push_back(col);
          for (size_t i = 0; i < rb * cb; ++i) {
            double t = col == t_col ? t_block[i] : 0.0;
            o.vals.push_back(t - omega * scaled[i]);
          }
          ++n;
        });
        o.lengths.push_back(n);
      }
    });
    stitch(out, rows, rb, cb, prolongator);
    tentative = Bsr();
    phase = PRODUCT;
  }

  // A P row by row (transfer.rs:155-169).
  void run_product() {
    size_t rb = current.rb, cb = MODES, rows = current.rows;
    int chunks = (rows < 4096 || opt.threads <= 1) ? 1 : opt.threads;
    vector<RowChunk> out(chunks);
    chunked(rows, opt.threads, [&](int ci, size_t b, size_t e) {
      RowAccumulator acc(aggregates, rb * cb);
      RowChunk& o = out[ci];
      for (size_t row = b; row < e; ++row) {
        acc.begin();
        for (uint32_t at = current.starts[row]; at < current.starts[row + 1]; ++at) {
          uint32_t col = current.cols[at];
          for (uint32_t in = prolongator.starts[col]; in < prolongator.starts[col + 1]; ++in)
            add_product(acc.entry(prolongator.cols[in]), current.block(at), rb, current.cb, prolongator.block(in), cb);
        }
        uint32_t n = 0;
        acc.drain([&](uint32_t col, const double* blk) {
          o.cols.push_back(col);
          o.vals.insert(o.vals.end(), blk, blk + rb * cb);
          ++n;
        });
        o.lengths.push_back(n);
      }
    });
    stitch(out, rows, rb, cb, ap);
    phase = GALERKIN;
  }

  // P^T (A P) by coarse row, P read by columns with fine rows ascending (transfer.rs:173-238).
  void run_galerkin() {
    size_t fine = prolongator.rb, cdim = MODES;
    vector<uint32_t> cstarts(aggregates + 1, 0);
    for (uint32_t c : prolongator.cols) cstarts[c + 1] += 1;
    for (size_t i = 0; i < aggregates; ++i) cstarts[i + 1] += cstarts[i];
    vector<uint32_t> filled(cstarts.begin(), cstarts.end() - 1);
    vector<std::pair<uint32_t, uint32_t>> entries(prolongator.cols.size());
    for (size_t row = 0; row < prolongator.rows; ++row)
      for (uint32_t at = prolongator.starts[row]; at < prolongator.starts[row + 1]; ++at)
        entries[filled[prolongator.cols[at]]++] = {(uint32_t)row, at};
    int chunks = (aggregates < 4096 || opt.threads <= 1) ? 1 : opt.threads;
    vector<RowChunk> out(chunks);
    chunked(aggregates, opt.threads, [&](int ci, size_t b, size_t e) {
      RowAccumulator acc(aggregates, cdim * cdim);
      RowChunk& o = out[ci];
      vector<double> tr(fine * cdim);
      for (size_t c = b; c < e; ++c) {
        acc.begin();
        for (uint32_t k = cstarts[c]; k < cstarts[c + 1]; ++k) {
          uint32_t fine_row = entries[k].first;
          const double* blk = prolongator.block(entries[k].second);
          for (size_t p = 0; p < fine; ++p)
            for (size_t q = 0; q < cdim; ++q) tr[q * fine + p] = blk[p * cdim + q];
          for (uint32_t in = ap.starts[fine_row]; in < ap.starts[fine_row + 1]; ++in)
            add_product(acc.entry(ap.cols[in]), tr.data(), cdim, fine, ap.block(in), cdim);
        }
        uint32_t n = 0;
        acc.drain([&](uint32_t col, const double* blk) {
          o.cols.push_back(col);
          o.vals.insert(o.vals.end(), blk, blk + cdim * cdim);
          ++n;
        });
        o.lengths.push_back(n);
      }
    });
    stitch(out, aggregates, cdim, cdim, coarse);
    // finish_level, setup.rs:650-695: a zero coarse diagonal becomes one.
    for (size_t row = 0; row < coarse.rows; ++row)
      for (uint32_t at = coarse.starts[row]; at < coarse.starts[row + 1]; ++at) {
        if (coarse.cols[at] != row) continue;
        for (size_t d = 0; d < cdim; ++d) {
          double& v = coarse.vals[(size_t)at * 36 + d * cdim + d];
          if (v == 0.0) v = 1.0;
        }
      }
    HostLevel lv;
    lv.a = std::move(current);
    lv.inverse_diagonal = std::move(inv);
    lv.lambda_max = lambda_max;
    lv.lambda_min = lambda_max / opt.range;
    lv.has_p = true;
    lv.p = std::move(prolongator);
    lv.aggregates = std::move(aggregate);
    levels.push_back(std::move(lv));
    current = std::move(coarse);
    coarse = Bsr();
    ap = Bsr();
    near_null = std::move(coarse_null);
    positions = std::move(coarse_positions);
    reach = opt.reach;
    retries = 0;
    is_coarsest = false;
    aggregates = 0;
    phase = DIAGONAL;
  }

  void push_final(bool factored) {
    HostLevel lv;
    lv.a = std::move(current);
    lv.inverse_diagonal = std::move(inv);
    lv.lambda_max = lambda_max;
    lv.lambda_min = lambda_max / opt.range;
    lv.has_factor = factored;
    levels.push_back(std::move(lv));
  }

  // Dense Cholesky of the coarsest level (block.rs:307-374), then its explicit inverse
  // L^-T L^-1, which the device applies as one matrix-vector product per cycle.
  sf_status run_factor() {
    size_t n = current.rows * current.rb;
    vector<double> f(n * n, 0.0);
    for (size_t row = 0; row < current.rows; ++row)
      for (uint32_t at = current.starts[row]; at < current.starts[row + 1]; ++at) {
        size_t col = current.cols[at];
        for (size_t p = 0; p < current.rb; ++p)
          for (size_t q = 0; q < current.cb; ++q)
            f[(row * current.rb + p) * n + col * current.cb + q] = current.block(at)[p * current.cb + q];
      }
    for (size_t j = 0; j < n; ++j) {
      double sum = f[j * n + j];
      for (size_t k = 0; k < j; ++k) sum -= f[j * n + k] * f[j * n + k];
      if (!std::isfinite(sum) || sum <= 0.0) return fail_pd(j, sum);
      double d = std::sqrt(sum);
      f[j * n + j] = d;
      rows_parallel(n - j - 1, opt.threads, [&](size_t o) {
        size_t i = j + 1 + o;
        double s = f[i * n + j];
        for (size_t k = 0; k < j; ++k) s -= f[i * n + k] * f[j * n + k];
        f[i * n + j] = s / d;
      });
    }
    // L^-1 column by column (forward substitution on unit vectors), then A^-1 = L^-T L^-1.
    vector<double> li(n * n, 0.0);
    rows_parallel(n, opt.threads, [&](size_t c) {
      for (size_t i = c; i < n; ++i) {
        double s = i == c ? 1.0 : 0.0;
        for (size_t k = c; k < i; ++k) s -= f[i * n + k] * li[k * n + c];
        li[i * n + c] = s / f[i * n + i];
      }
    });
    HostLevel lv;
    lv.coarse_inverse.assign(n * n, 0.0);
    rows_parallel(n, opt.threads, [&](size_t i) {
      for (size_t j = 0; j < n; ++j) {
        double s = 0.0;
        for (size_t k = std::max(i, j); k < n; ++k) s += li[k * n + i] * li[k * n + j];
        lv.coarse_inverse[i * n + j] = s;
      }
    });
    lv.factor_n = n;
    lv.a = std::move(current);
    lv.inverse_diagonal = std::move(inv);
    lv.lambda_max = lambda_max;
    lv.lambda_min = lambda_max / opt.range;
    lv.has_factor = true;
    levels.push_back(std::move(lv));
    phase = DONE;
    return SF_OK;
  }
};

SetupMachine* setup_create(Bsr&& fine, vector<double>&& near_null, vector<P3>&& positions,
                           const SetupOptions& options) {
  SetupMachine* m = new SetupMachine;
  m->opt = options;
  m->current = std::move(fine);
  m->near_null = std::move(near_null);
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
      case STRENGTH: m->run_strength(); break;
      case AGGREGATE: m->run_aggregate(); break;
      case TENTATIVE: m->run_tentative(); break;
      case SPECTRAL: m->run_spectral(); rows *= 20; break;
      case FILTER: m->run_filter(); break;
      case SMOOTH: m->run_smooth(); break;
      case PRODUCT: m->run_product(); break;
      case GALERKIN: m->run_galerkin(); break;
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
