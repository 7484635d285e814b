// Mixed-precision CG (placeholder until the batched engine lands).
#include "hw_internal.h"

namespace hw {
int mixed_solve(const hw_gauge *, double, const hw_field *, hw_field *, int, const hw_cg_params &, hw_cg_result *) {
    set_error("mixed-precision solve is not available in this build");
    return HW_ERR_INVALID;
}
}  // namespace hw
