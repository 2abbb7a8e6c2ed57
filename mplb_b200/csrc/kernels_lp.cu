// Shifted FP32 and FP16-storage instantiations (FP32 arithmetic, fused
// multiply-adds allowed).
#include "launch_impl.cuh"

namespace mplb {

template struct Launch<2, float>;
template struct Launch<3, float>;
template struct Launch<2, __half>;
template struct Launch<3, __half>;

}  // namespace mplb

#include "batch_kernels.cuh"

namespace mplb {

template struct BatchLaunch<float>;

}  // namespace mplb
