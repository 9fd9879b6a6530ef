// VAJRA_ALGO_HALPERN (placeholder until the restarted Halpern driver lands).
#include "solver.cuh"

namespace vajra {
vajra_status run_halpern(vajra_pdhg* h, vajra_result* r) {
    (void)h; (void)r;
    set_error("HALPERN driver not built yet");
    return VAJRA_ERR_INTERNAL;
}
}  // namespace vajra
