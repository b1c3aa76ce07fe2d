// The serving loop: solve requests arrive at any time, are admitted in arrival order while their
// estimated device memory fits the budget, are built on host worker threads (each study on its own
// CUDA stream), and are solved with their hierarchy and vectors resident on the device.
//
// Continuous batching: a study with fewer free DOFs than `batch_max_dofs` is built `batchable`
// and handed to the batch thread, which keeps one batch per launch signature (studies of the same
// depth share one). Between chunks of iterations a batch drops the studies that have stopped and
// takes in the ones that became ready meanwhile, so requests that arrive while others are on the
// GPU join as slots and memory free up; each step of a batch is one grid per kernel over all its
// studies. Larger studies go to solver threads and solve on their own streams, overlapping on the
// device with the batches and with each other while the build workers go on building.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "batch.h"
#include "sf_internal.h"

namespace sf {

namespace {

const uint64_t kBytesPerDofEstimate = 6144;  // admission estimate before a study is built

struct Request {
  uint64_t id = 0;
  sf_model* model = nullptr;
  sf_study_options options;
  uint64_t free_dofs = 0, node_count = 0;
  uint64_t reserved = 0;  // bytes held against the budget
  bool batchable = false;
  double t_submit = 0, t_admit = 0, t_built = 0, t_done = 0;
  sf_study* study = nullptr;
  int state = 0;  // 0 pending, 1 building, 2 solving, 3 done
  sf_status status = SF_OK;
  sf_step_outcome outcome{};
  std::vector<double> displacements;
  uint64_t device_bytes = 0;
  uint64_t batch_peak = 0;  // the largest batch it ran in
  char message[160] = {0};  // the failure's message
  std::atomic<bool> cancel{false};  // sf_server_cancel asked for it
};

// The cancel callback of a request's build and solve.
int32_t request_cancelled(void* user) { return static_cast<Request*>(user)->cancel.load() ? 1 : 0; }

}  // namespace

}  // namespace sf

struct sf_server {
  sf_server_options opt;
  std::mutex m;
  std::condition_variable cv;
  bool stopping = false;
  uint64_t next_id = 1;
  uint64_t reserved = 0, peak_reserved = 0;
  std::deque<sf::Request*> pending;      // submitted, not admitted
  std::deque<sf::Request*> admitted;     // waiting for a build worker
  std::vector<sf::Request*> ready;       // built, batchable, waiting for a batch
  std::deque<sf::Request*> solving;      // built, too large to batch, waiting for a solver thread
  uint64_t building = 0;                 // requests inside a build worker
  std::unordered_map<uint64_t, std::unique_ptr<sf::Request>> all;
  std::vector<std::thread> workers, solvers;
  std::thread batcher;
  uint64_t completed = 0, batches_run = 0, batched_requests = 0, batch_member_sum = 0, batch_chunks = 0;
  std::unordered_map<sf_study*, sf::Request*> owners;  // batch thread only

  // Admits pending requests in arrival order while they fit the budget. Caller holds m.
  void admit_locked() {
    while (!pending.empty()) {
      sf::Request* r = pending.front();
      uint64_t need = r->free_dofs * sf::kBytesPerDofEstimate;
      if (reserved > 0 && reserved + need > opt.memory_budget) break;
      pending.pop_front();
      r->reserved = need;
      reserved += need;
      peak_reserved = std::max(peak_reserved, reserved);
      r->t_admit = sf::now_seconds();
      r->state = 1;
      admitted.push_back(r);
    }
  }

  // Records a finished request: its displacements to the host, the study released. Caller does
  // not hold m.
  void complete(sf::Request* r, sf_status st) {
    if (st) {
      sf_error err;
      sf_last_error(&err);
      std::snprintf(r->message, sizeof r->message, "%.159s", err.message);
    }
    if (r->study) {
      if (!st) {
        r->displacements.assign(r->node_count * 3, 0.0);
        sf_status e = sf_study_displacements(r->study, r->displacements.data());
        if (e) st = e;
      }
      sf_study_destroy(r->study);
      r->study = nullptr;
    }
    std::lock_guard<std::mutex> lock(m);
    r->status = st;
    r->t_done = sf::now_seconds();
    r->state = 3;
    reserved -= r->reserved;
    r->reserved = 0;
    ++completed;
    admit_locked();
    cv.notify_all();
  }

  void worker_loop() {
    for (;;) {
      sf::Request* r = nullptr;
      {
        std::unique_lock<std::mutex> lock(m);
        cv.wait(lock, [&] { return stopping || !admitted.empty(); });
        if (admitted.empty()) return;
        r = admitted.front();
        admitted.pop_front();
        ++building;
      }
      sf_study* st = nullptr;
      sf_model* model = r->model;
      r->model = nullptr;
      sf_status e = sf_study_create(model, &r->options, sf::request_cancelled, r, &st);
      r->t_built = sf::now_seconds();
      if (e) {
        {
          std::lock_guard<std::mutex> lock(m);
          --building;
        }
        complete(r, e);
        continue;
      }
      r->study = st;
      r->device_bytes = sf::study_device_bytes(st);
      {
        // The budget now holds the study's real footprint.
        std::lock_guard<std::mutex> lock(m);
        --building;
        reserved = reserved - r->reserved + r->device_bytes;
        peak_reserved = std::max(peak_reserved, reserved);
        r->reserved = r->device_bytes;
        admit_locked();
        r->state = 2;
        if (r->batchable)
          ready.push_back(r);
        else
          solving.push_back(r);
      }
      cv.notify_all();
    }
  }

  // Solves built studies too large to batch, each on its own stream, so the build workers keep
  // building meanwhile; several solver threads overlap their studies on the device.
  void solver_loop() {
    for (;;) {
      sf::Request* r = nullptr;
      {
        std::unique_lock<std::mutex> lock(m);
        cv.wait(lock, [&] { return (stopping && admitted.empty() && building == 0) || !solving.empty(); });
        if (solving.empty()) return;
        r = solving.front();
        solving.pop_front();
      }
      sf_step_outcome out{};
      sf_status e = sf_study_step(r->study, UINT64_MAX, sf::request_cancelled, r, &out);
      r->outcome = out;
      if (!e && out.kind == SF_OUTCOME_CANCELLED) e = sf::fail(SF_CANCELLED, "the request was cancelled");
      complete(r, e);
    }
  }

  // Members of a batch whose requests were cancelled leave it between chunks; the others go on.
  void drop_cancelled(sf::BatchRunner& run) {
    std::vector<sf_study*> keep;
    for (sf_study* st : run.members) {
      sf::Request* r = owners[st];
      if (!r->cancel.load()) {
        keep.push_back(st);
        continue;
      }
      owners.erase(st);
      run.dirty = true;
      complete(r, sf::fail(SF_CANCELLED, "the request was cancelled"));
    }
    run.members.swap(keep);
  }

  void batch_loop() {
    std::map<uint64_t, std::unique_ptr<sf::BatchRunner>> runners;
    uint64_t chunk = 8;
    for (;;) {
      std::vector<sf::Request*> joining;
      {
        std::unique_lock<std::mutex> lock(m);
        bool busy = false;
        for (auto& kv : runners) busy = busy || !kv.second->members.empty();
        cv.wait(lock, [&] { return stopping || !ready.empty() || busy; });
        if (stopping && ready.empty() && !busy && admitted.empty() && building == 0) return;
        joining.swap(ready);
      }
      for (sf::Request* r : joining) {
        if (r->cancel.load()) {
          complete(r, sf::fail(SF_CANCELLED, "the request was cancelled"));
          continue;
        }
        uint64_t sig = sf::study_signature(r->study);
        auto& run = runners[sig];
        if (!run) {
          run.reset(new sf::BatchRunner);
          if (sf_status e = run->init(opt.device)) {
            complete(r, e);
            continue;
          }
        }
        if (sf_status e = sf_study_resolve(r->study, nullptr)) {
          complete(r, e);
          continue;
        }
        cudaStreamSynchronize((cudaStream_t)(uintptr_t)sf_study_stream(r->study));
        run->members.push_back(r->study);
        run->dirty = true;
        owners[r->study] = r;
      }
      for (auto& kv : runners) {
        sf::BatchRunner& run = *kv.second;
        drop_cancelled(run);
        if (run.members.empty()) continue;
        // A batch holds at most max_batch studies; the rest wait in the ready list.
        if (run.members.size() > opt.max_batch) {
          std::lock_guard<std::mutex> lock(m);
          while (run.members.size() > opt.max_batch) {
            ready.push_back(owners[run.members.back()]);
            run.members.pop_back();
          }
        }
        if (run.dirty) ++batches_run;
        std::vector<sf_study*> finished;
        size_t size = run.members.size();
        for (sf_study* s : run.members) {
          sf::Request* r = owners[s];
          r->batch_peak = std::max<uint64_t>(r->batch_peak, size);
        }
        ++batch_chunks;
        batch_member_sum += size;
        sf_status e = run.run_chunk(chunk, finished);
        if (e) {
          // A batch that cannot run fails its members.
          for (sf_study* s : run.members) finished.push_back(s);
          run.members.clear();
          run.dirty = true;
        }
        for (sf_study* s : finished) {
          sf::Request* r = owners[s];
          sf_status st = e;
          if (!e) {
            sf_step_outcome out{};
            st = sf_study_step(s, 0, nullptr, nullptr, &out);
            r->outcome = out;
          }
          {
            std::lock_guard<std::mutex> lock(m);
            ++batched_requests;
          }
          owners.erase(s);
          complete(r, st);
        }
      }
    }
  }

};

extern "C" {

void sf_server_options_default(sf_server_options* o) {
  if (!o) return;
  o->device = 0;
  o->memory_budget = 150ull << 30;
  o->batch_max_dofs = 100000;
  o->max_batch = 64;
  o->build_threads = 8;
  o->solve_threads = 4;
  o->setup_threads = 2;
}

sf_status sf_server_create(const sf_server_options* options, sf_server** out) {
  if (!out) return sf::fail(SF_INVALID_ARGUMENT, "null argument");
  std::unique_ptr<sf_server> s(new sf_server);
  sf_server_options_default(&s->opt);
  if (options) s->opt = *options;
  if (s->opt.memory_budget == 0) s->opt.memory_budget = 150ull << 30;
  if (s->opt.max_batch == 0) s->opt.max_batch = 64;
  if (s->opt.build_threads == 0) s->opt.build_threads = 8;
  if (s->opt.solve_threads == 0) s->opt.solve_threads = 4;
  if (s->opt.setup_threads == 0) s->opt.setup_threads = 2;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return sf::fail(SF_NO_DEVICE, "no CUDA device is visible");
  if (s->opt.device < 0 || s->opt.device >= ndev) return sf::fail(SF_INVALID_ARGUMENT, "no such CUDA device");
  sf_server* raw = s.get();
  for (uint64_t i = 0; i < s->opt.build_threads; ++i)
    s->workers.emplace_back([raw] {
      cudaSetDevice(raw->opt.device);
      raw->worker_loop();
    });
  for (uint64_t i = 0; i < s->opt.solve_threads; ++i)
    s->solvers.emplace_back([raw] {
      cudaSetDevice(raw->opt.device);
      raw->solver_loop();
    });
  s->batcher = std::thread([raw] {
    cudaSetDevice(raw->opt.device);
    raw->batch_loop();
  });
  *out = s.release();
  return SF_OK;
}

sf_status sf_server_submit(sf_server* s, sf_model* model, const sf_study_options* options, uint64_t* id) {
  if (!s || !model || !options || !id) {
    if (model) sf_model_destroy(model);
    return sf::fail(SF_INVALID_ARGUMENT, "null argument");
  }
  std::unique_ptr<sf::Request> r(new sf::Request);
  r->options = *options;
  r->options.device = s->opt.device;
  r->free_dofs = sf::model_free_dofs(model);
  r->node_count = sf::model_node_count(model);
  r->batchable = r->options.preconditioner == SF_PRECONDITIONER_MULTIGRID && r->free_dofs < s->opt.batch_max_dofs;
  if (r->batchable) r->options.batchable = 1;
  if (r->options.threads == 0) r->options.threads = s->opt.setup_threads;
  r->model = model;
  r->t_submit = sf::now_seconds();
  std::lock_guard<std::mutex> lock(s->m);
  if (s->stopping) {
    sf_model_destroy(r->model);
    return sf::fail(SF_INVALID_ARGUMENT, "the server is shutting down");
  }
  r->id = s->next_id++;
  *id = r->id;
  s->pending.push_back(r.get());
  s->all[r->id] = std::move(r);
  s->admit_locked();
  s->cv.notify_all();
  return SF_OK;
}

sf_status sf_server_wait(sf_server* s, uint64_t id, uint64_t timeout_ms, sf_request_result* out) {
  if (!s) return sf::fail(SF_INVALID_ARGUMENT, "null argument");
  std::unique_lock<std::mutex> lock(s->m);
  auto it = s->all.find(id);
  if (it == s->all.end()) return sf::fail(SF_INVALID_ARGUMENT, "no such request");
  sf::Request* r = it->second.get();
  auto done = [&] { return r->state == 3; };
  if (timeout_ms == UINT64_MAX)
    s->cv.wait(lock, done);
  else
    s->cv.wait_for(lock, std::chrono::milliseconds(timeout_ms), done);
  if (out) {
    std::memset(out, 0, sizeof(*out));
    out->status = r->status;
    out->finished = r->state == 3;
    out->batched = r->batchable;
    out->batch_size = r->batch_peak;
    out->outcome = r->outcome;
    out->free_dofs = r->free_dofs;
    out->node_count = r->node_count;
    out->device_bytes = r->device_bytes;
    double end = r->state == 3 ? r->t_done : sf::now_seconds();
    out->queue_seconds = (r->t_admit ? r->t_admit : end) - r->t_submit;
    out->build_seconds = r->t_built ? r->t_built - r->t_admit : 0.0;
    out->solve_seconds = r->state == 3 && r->t_built ? r->t_done - r->t_built : 0.0;
    out->latency_seconds = end - r->t_submit;
    std::snprintf(out->message, sizeof out->message, "%s", r->message);
  }
  if (r->state != 3) return sf::fail(SF_NOT_FINISHED, "the request is still running");
  return SF_OK;
}

sf_status sf_server_take(sf_server* s, uint64_t id, double* displacements) {
  if (!s) return sf::fail(SF_INVALID_ARGUMENT, "null argument");
  std::unique_ptr<sf::Request> r;
  {
    std::lock_guard<std::mutex> lock(s->m);
    auto it = s->all.find(id);
    if (it == s->all.end()) return sf::fail(SF_INVALID_ARGUMENT, "no such request");
    if (it->second->state != 3) return sf::fail(SF_NOT_FINISHED, "the request is still running");
    r = std::move(it->second);
    s->all.erase(it);
  }
  if (r->status) return sf::fail(r->status, "the request failed");
  if (displacements) std::memcpy(displacements, r->displacements.data(), r->displacements.size() * 8);
  return SF_OK;
}

sf_status sf_server_cancel(sf_server* s, uint64_t id) {
  if (!s) return sf::fail(SF_INVALID_ARGUMENT, "null argument");
  sf::Request* dropped = nullptr;
  {
    std::lock_guard<std::mutex> lock(s->m);
    auto it = s->all.find(id);
    if (it == s->all.end()) return sf::fail(SF_INVALID_ARGUMENT, "no such request");
    sf::Request* r = it->second.get();
    if (r->state == 3) return SF_OK;  // finished already: nothing to cancel
    r->cancel.store(true);
    // Not yet taken by a worker: it leaves the queue here. Later stages read the flag.
    for (auto* q : {&s->pending, &s->admitted}) {
      auto at = std::find(q->begin(), q->end(), r);
      if (at != q->end()) {
        q->erase(at);
        dropped = r;
        break;
      }
    }
  }
  if (dropped) {
    if (dropped->model) {
      sf_model_destroy(dropped->model);
      dropped->model = nullptr;
    }
    s->complete(dropped, sf::fail(SF_CANCELLED, "the request was cancelled"));
  }
  return SF_OK;
}

sf_status sf_server_statistics(sf_server* s, sf_server_stats* out) {
  if (!s || !out) return sf::fail(SF_INVALID_ARGUMENT, "null argument");
  std::lock_guard<std::mutex> lock(s->m);
  std::memset(out, 0, sizeof(*out));
  out->completed = s->completed;
  out->pending = s->pending.size();
  out->reserved_bytes = s->reserved;
  out->peak_reserved_bytes = s->peak_reserved;
  out->batches = s->batches_run;
  out->batched_requests = s->batched_requests;
  out->mean_batch_size = s->batch_chunks ? (double)s->batch_member_sum / (double)s->batch_chunks : 0.0;
  return SF_OK;
}

void sf_server_destroy(sf_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lock(s->m);
    s->stopping = true;
    s->cv.notify_all();
  }
  for (auto& t : s->workers) t.join();
  {
    std::lock_guard<std::mutex> lock(s->m);
    s->cv.notify_all();
  }
  for (auto& t : s->solvers) t.join();
  if (s->batcher.joinable()) s->batcher.join();
  for (auto& kv : s->all) {
    if (kv.second->model) sf_model_destroy(kv.second->model);
    if (kv.second->study) sf_study_destroy(kv.second->study);
  }
  delete s;
}

}  // extern "C"
