// Batched solves and the serving loop's view of a study (study.cpp, server.cpp).
#pragma once

#include <cstdint>
#include <vector>

#include "device.h"

namespace sf {

// Several resident studies advanced together on one stream: each conjugate gradient step of all
// members is one captured graph whose kernels are single grids over the members (blockIdx.y =
// member), each masked by its own status word. Membership changes (finished members leave, new
// ones join) rebuild the graph between chunks.
struct BatchRunner {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<sf_study*> members;
  BatchIteration it;
  std::vector<void*> slots;  // pinned slots for the members' states
  bool dirty = true;

  ~BatchRunner();
  sf_status init(int device);
  sf_status rebuild();
  // Replays `iterations` batched iterations, reads every member's state and moves the members
  // that stopped (converged or failed) into `finished`.
  sf_status run_chunk(uint64_t iterations, std::vector<sf_study*>& finished);
};

// A hash of the kernels one iteration of the study launches: studies with equal signatures can
// share a batch.
uint64_t study_signature(sf_study* s);
uint64_t study_device_bytes(const sf_study* s);
// Free DOFs and nodes of a model before it is built.
uint64_t model_free_dofs(const sf_model* m);
uint64_t model_node_count(const sf_model* m);

}  // namespace sf
