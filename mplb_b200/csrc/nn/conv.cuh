// Implicit-GEMM 2D convolutions on the 5th-generation tensor cores.
//
// Activations are NHWC bf16 "views": a base pointer, a pixel stride (elements
// between consecutive pixels, >= channels, a multiple of 8) and a channel
// count, so a convolution can read or write a channel slice of a wider
// (concatenated) buffer.  Weights are bf16 [cout][taps][cin] (taps = 9 for a
// 3x3 kernel with one pixel of zero padding, 1 for 1x1).
//
// ConvKernel computes, for a tile of 128 consecutive pixels (M) and `bn`
// output channels (N), D = sum over taps t and input channels c of
// X[pixel + offset(t)][c] * Wt[n][t][c] (K = taps * cin), with the pixels of
// the tile fetched by one TMA box per k-block: box (BK channels, W pixels,
// 128 / W rows) at the tap's shifted coordinates, whose out-of-image parts
// TMA fills with zeros (the padding).  A and B are K-major, swizzled by BK * 2
// bytes; the accumulator lives in TMEM (128 lanes x bn fp32 columns).  The
// same kernel is the data gradient of a convolution when it is given the
// output gradient as X and the flipped, transposed weights
// W'[c][8 - t][n] = W[n][t][c].
//
// WgradKernel computes dW[n][t][c] += sum over pixels p of dY[p][n] *
// X[p + offset(t)][c]: M = 128 output channels, N = input channels, K = a
// range of 128-pixel blocks (split over CTAs, accumulated with fp32 atomics).
// Both operands arrive pixel-major with channels contiguous, i.e. MN-major,
// as 64-channel TMA boxes swizzled by 128 bytes.
//
// Warp roles (128 threads): warp 0 issues TMA loads, warp 1 issues MMAs,
// warp 2 owns the TMEM allocation, all four warps run the epilogue (warp w
// reads TMEM lanes 32w..32w+31).  Barrier waits are bounded; a CTA that
// gives up sets `err` and skips its stores.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>

namespace mplb {
namespace nn {

constexpr int kConvThreads = 128;
constexpr int kTileM = 128;

struct ConvArgs {
    int H, W;              // image size in pixels
    int tiles_per_img;     // H * W / 128
    int bh;                // image rows per 128-pixel tile (128 / W)
    int cin;               // channels of the input view (K per tap, padded
                           // to BK with zeros by the tensor map)
    int taps;              // 9 or 1
    int nkb;               // k-blocks: taps * ceil(cin / BK)
    int cout;              // valid output channels
    int bn;                // UMMA N of one CTA
    int stages;            // pipeline depth
    int tmem_cols;         // TMEM columns allocated (power of two >= bn)
    // epilogue
    void* out;             // bf16 or fp32 view
    long long out_ps;      // pixel stride of out (elements)
    int out_coff;          // channel offset of out
    int out_f32;           // 1: fp32 output, 0: bf16
    const float* bias;     // per output channel, or null
    int relu;              // apply max(0, .)
    const __nv_bfloat16* mask;   // multiply by (mask > 0), or null
    long long mask_ps;
    int mask_coff;
    int* err;              // set to 1 when a wait gives up
};

struct WgradArgs {
    int H, W, tiles_per_img, bh;
    int taps;
    int cout, cin;         // dW is [cout][taps][cin]
    int bn;                // UMMA N: 64 * b_atoms
    int b_atoms;           // 64-channel boxes of X per stage (<= 4)
    int kb_total;          // 128-pixel blocks in the batch
    int kb_per_split;
    int stages;
    int tmem_cols;
    float* dw;
    int* err;
};

// Weight gradient of layers with few output channels (cout <= 64), with the
// roles of the operands swapped: M = 128 rows of (tap, 32-channel chunk of
// the input) pairs - four "atoms", each one 32-channel TMA box of X at its
// tap's shifted coordinates - N = the output channels (32 or 64, from
// 32-channel boxes of dY), K = 128-pixel blocks split over CTAs.  Both
// operands MN-major, swizzled by 64 bytes.  Padding M to 128 for 32 output
// channels and N to 64 for 32 input channels, as WgradKernel does for
// these layers, wasted 7/8 of the tensor work.
struct WgradTArgs {
    int H, W, tiles_per_img, bh;
    int taps;
    int cout, cin;         // dW is [cout][taps][cin]
    int ci_chunks;         // 32-channel chunks of the input
    int n_atoms;           // taps * ci_chunks
    int bn;                // UMMA N: 32 * ceil(cout / 32)
    int kb_total;          // 128-pixel blocks in the batch
    int kb_per_split;
    int stages;
    int tmem_cols;
    float* dw;
    int* err;
};

template <int BK>
__global__ void ConvKernel(const __grid_constant__ CUtensorMap ta,
                           const __grid_constant__ CUtensorMap tb,
                           ConvArgs a);

__global__ void WgradTKernel(const __grid_constant__ CUtensorMap tx,
                             const __grid_constant__ CUtensorMap tdy,
                             WgradTArgs a);

__global__ void WgradKernel(const __grid_constant__ CUtensorMap ta,
                            const __grid_constant__ CUtensorMap tb,
                            WgradArgs a);

// Shared memory a launch needs (stage buffers + 1 KiB alignment slack +
// barriers).
inline int ConvSmemBytes(int bk, int bn, int stages) {
    return 1024 + stages * (kTileM * bk * 2 + bn * bk * 2) + 256;
}
inline int WgradSmemBytes(int b_atoms, int stages) {
    return 1024 + stages * ((2 + b_atoms) * 16384) + 256;
}
// WgradTKernel: per stage four 8 KiB X atoms and bn / 32 8 KiB dY atoms.
inline int WgradTSmemBytes(int bn, int stages) {
    return 1024 + stages * ((4 + bn / 32) * 8192) + 256;
}

}  // namespace nn
}  // namespace mplb
