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
};
