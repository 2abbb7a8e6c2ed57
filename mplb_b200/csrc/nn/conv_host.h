// Host launchers of the tensor-core convolution kernels.
#pragma once

#include <cuda_runtime.h>

#include <string>

namespace mplb {
namespace nn {

// A bf16 NHWC view (channel 0 of pixel 0 at ptr; pixels ps elements apart).
struct View {
    void* ptr;
    int nimg, h, w, c;
    long long ps;
};

// y = act(conv(x, w) + bias) [* (mask > 0)]; false (with err) on a rejected
// shape or launch.  err_dev: device word the kernel sets on a timed-out wait.
bool LaunchConv(const View& x, const void* w, int taps, const float* bias,
                int relu, const View& y, bool y_f32, const View* mask,
                cudaStream_t stream, int* err_dev, std::string& err);

// dw[n][t][c] += sum_p dy[p][n] x[p + offset(t)][c].
bool LaunchWgrad(const View& dy, const View& x, int taps, float* dw,
                 int sm_count, cudaStream_t stream, int* err_dev,
                 std::string& err);

}  // namespace nn
}  // namespace mplb
