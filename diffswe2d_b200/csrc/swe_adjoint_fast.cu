// swe_adjoint_fast.cu -- the step adjoint's kernels (swe_adjoint_kernels.cuh)
// in the arithmetic of the tolerance-mode step (FastMath: rcp.approx,
// sqrt.approx, ex2/lg2.approx), compiled like swe_fast.cu (-fmad=true
// -ftz=true).  The C ABI (swe_adjoint.cu) runs these for parameters with
// arithmetic = SWE_ARITH_FAST: the gradient of a tolerance-mode run, within
// FP32 rounding of the IEEE adjoint.
#include "swe_adjoint_kernels.cuh"

namespace swe {

int fast_launch_adj_spatial(const AdjArgs& a, int level_blocks, bool pred, cudaStream_t s) {
    return launch_adj_spatial<FastMath>(a, level_blocks, pred, s);
}

int fast_launch_adj_pointwise(const PwArgs& a, cudaStream_t s) {
    return launch_adj_pointwise<FastMath>(a, s);
}

}  // namespace swe
