// Path-tracing passes (placeholder until the wavefront tracer lands).
#include "tracer.h"

namespace pfxt {

void trace_sample(pfxt_trace& t, uint32_t count, uint32_t seed) {
  (void)t;
  (void)count;
  (void)seed;
  throw Invalid("sampling is not built yet");
}

void trace_sample_adaptive(pfxt_trace& t, const pfxt_adaptive& a, uint32_t seed, pfxt_round* rounds, uint32_t cap,
                           uint32_t* written) {
  (void)t;
  (void)a;
  (void)seed;
  (void)rounds;
  (void)cap;
  (void)written;
  throw Invalid("sampling is not built yet");
}

}  // namespace pfxt
