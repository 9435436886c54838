// Learned-gauge predictor (placeholder until the network kernels land).
#include "pond_internal.h"

namespace pond {
int run_predictor(pond_ctx* c) {
  (void)c;
  return set_error(POND_ERR_UNSUPPORTED, "learned gauge predictor not built");
}
}  // namespace pond
