// Tensor-core mixed-precision path (placeholder until the tcgen05 kernels land).
#include "icc_device.cuh"

namespace icc {

void mixed_release(Op &) {}
int mixed_on_scale_update(Op &) { return ICC_OK; }
int mixed_solve(Op &, const double *, const double *, double, int64_t, const icc_solve_opts &, double *, int64_t *,
                double *) {
    return set_error(ICC_BAD_ARG, "ICC_MIXED is not available in this build");
}

}  // namespace icc
