// NTT tile-shape autotuner (autotune.cu).
#pragma once
#include "context.hpp"

namespace fides {
// Times every supported tile shape per (direction, pass, launch-size class) and stores the
// fastest in c->ntt_g.  best_ms (optional, 8 entries: [inverse][size class]) receives the
// time of one transform of the class's representative launch with the chosen shapes.
void autotune_ntt(Context* c, float* best_ms);
}  // namespace fides
