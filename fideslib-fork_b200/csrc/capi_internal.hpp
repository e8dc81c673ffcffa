// The opaque handle behind fides_ctx* (include/fides_b200.h), shared by the C-ABI files.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "context.hpp"

namespace fides {
// Sets the calling thread's message returned by fides_last_error().
void set_last_error(const std::string& msg);
}  // namespace fides

struct fides_ctx {
  fides::Context* c;
  cudaStream_t host_stream;  // stream of the host-buffer entry points (and pipelined compute)
  cudaStream_t h2d_stream = nullptr;  // pipelined host batches: host -> device copies
  cudaStream_t d2h_stream = nullptr;  //                         device -> host copies
  // Pipelined host batches keep their device slots and events between calls, so that calls
  // that return before completion (fides_*_host_batch_async) continue one pipeline: a slot is
  // reused once its previous item's device -> host copies are done, whichever call that was.
  static constexpr int kPipeSlots = 3;
  void* pipe_mem = nullptr;      // kPipeSlots slots of pipe_slot_bytes each
  size_t pipe_slot_bytes = 0;
  cudaEvent_t pipe_free[kPipeSlots] = {};      // recorded after a slot's device -> host copies
  cudaEvent_t pipe_in_ready[kPipeSlots] = {};  // after its host -> device copies
  cudaEvent_t pipe_computed[kPipeSlots] = {};  // after its computation
  bool pipe_used[kPipeSlots] = {};
  long pipe_next = 0;
};
