// Tensor-core convolution kernels (see conv.cuh for the formulation).
#include "conv.cuh"
#include "umma.cuh"

namespace mplb {
namespace nn {

using namespace umma;

namespace {

__device__ __forceinline__ uint8_t* Align1024(uint8_t* p) {
    const uint32_t s = SmemAddr(p);
    return p + ((1024u - (s & 1023u)) & 1023u);
}

__device__ __forceinline__ void Flag(volatile int* cta_err, int* err) {
    *cta_err = 1;
    atomicExch(err, 1);
}

__device__ __forceinline__ uint32_t PackBf16(float lo, float hi) {
    __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&h);
}

__device__ __forceinline__ void TapOffset(int taps, int t, int& dh, int& dw) {
    dh = 0;
    dw = 0;
    if (taps == 9) {
        dh = t / 3 - 1;
        dw = t % 3 - 1;
    }
}

}  // namespace

template <int BK>
__global__ void __launch_bounds__(kConvThreads, 1)
    ConvKernel(const __grid_constant__ CUtensorMap ta,
               const __grid_constant__ CUtensorMap tb, ConvArgs a) {
    constexpr int SW = BK * 2;
    constexpr uint32_t A_BYTES = kTileM * BK * 2;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = Align1024(smem_raw);
    const uint32_t stage_bytes = A_BYTES + (uint32_t)a.bn * BK * 2;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + a.stages * stage_bytes);
    uint64_t* empty = full + a.stages;
    uint64_t* accum = empty + a.stages;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accum + 1);
    volatile int* cta_err = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mt = blockIdx.x;
    const int img = mt / a.tiles_per_img;
    const int h0 = (mt - img * a.tiles_per_img) * a.bh;
    const int n0 = blockIdx.y * a.bn;

    if (threadIdx.x == 0) {
        for (int s = 0; s < a.stages; s++) {
            BarInit(&full[s], 1);
            BarInit(&empty[s], 1);
        }
        BarInit(accum, 1);
        *cta_err = 0;
        FenceBarrierInit();
        PrefetchTmap(&ta);
        PrefetchTmap(&tb);
    }
    if (warp == 2) TmemAlloc(tmem_slot, a.tmem_cols);
    FenceBeforeSync();
    __syncthreads();
    FenceAfterSync();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // TMA producer
        const int c_per_tap = (a.cin + BK - 1) / BK;
        int kb = 0;
        for (; kb < a.nkb; kb++) {
            const int s = kb % a.stages;
            if (kb >= a.stages &&
                !BarWait(&empty[s], ((kb / a.stages) + 1) & 1, cta_err)) {
                Flag(cta_err, a.err);
                break;
            }
            const int t = kb / c_per_tap;
            const int c0 = (kb - t * c_per_tap) * BK;
            int dh, dw;
            TapOffset(a.taps, t, dh, dw);
            uint8_t* sa = smem + s * stage_bytes;
            BarArriveExpectTx(&full[s], stage_bytes);
            TmaLoad4D(sa, &ta, &full[s], c0, dw, h0 + dh, img);
            TmaLoad2D(sa + A_BYTES, &tb, &full[s], t * a.cin + c0, n0);
        }
        // the copies of the last stages issued must land before exit
        for (int j = kb > a.stages ? kb - a.stages : 0; j < kb; j++)
            if (!BarWaitDrain(&full[j % a.stages], (j / a.stages) & 1))
                Flag(cta_err, a.err);
    } else if (warp == 1 && lane == 0) {
        // MMA issuer
        const uint32_t idesc = InstrDescBf16(kTileM, a.bn, false, false);
        const uint32_t base = SmemAddr(smem);
        for (int kb = 0; kb < a.nkb; kb++) {
            const int s = kb % a.stages;
            if (!BarWait(&full[s], (kb / a.stages) & 1, cta_err)) {
                Flag(cta_err, a.err);
                break;
            }
            FenceAfterSync();
            const uint32_t sa = base + s * stage_bytes;
            const uint32_t sb = sa + A_BYTES;
#pragma unroll
            for (int k = 0; k < BK / 16; k++) {
                Mma(tmem, SmemDesc(sa + k * 32, 0, 8 * SW, SW),
                    SmemDesc(sb + k * 32, 0, 8 * SW, SW), idesc,
                    (kb | k) != 0 ? 1u : 0u);
            }
            Commit(&empty[s]);
        }
        Commit(accum);
    }
    __syncwarp();

    // Epilogue: TMEM lane = pixel row of the tile, column = output channel.
    const bool acc_ok = BarWaitDrain(accum, 0);
    FenceAfterSync();
    if (!acc_ok && threadIdx.x == 0) Flag(cta_err, a.err);
    const bool store = acc_ok && *cta_err == 0;
    const int row = warp * 32 + lane;
    const long long pix = (long long)mt * kTileM + row;
    for (int c = 0; c < a.bn; c += 16) {
        float v[16];
        TmemLoad16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
        const int n = n0 + c;
        if (!store || n >= a.cout) continue;
        if (a.bias != nullptr) {
            const float4* b4 = reinterpret_cast<const float4*>(a.bias + n);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const float4 b = b4[q];
                v[4 * q] += b.x;
                v[4 * q + 1] += b.y;
                v[4 * q + 2] += b.z;
                v[4 * q + 3] += b.w;
            }
        }
        if (a.relu) {
#pragma unroll
            for (int i = 0; i < 16; i++) v[i] = fmaxf(v[i], 0.0f);
        }
        if (a.mask != nullptr) {
            const uint4* m4 = reinterpret_cast<const uint4*>(
                a.mask + pix * a.mask_ps + a.mask_coff + n);
#pragma unroll
            for (int q = 0; q < 2; q++) {
                const uint4 m = m4[q];
                const uint32_t w[4] = {m.x, m.y, m.z, m.w};
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    // bf16 > 0: sign bit clear and not +0
                    if ((w[e] & 0x8000u) || (w[e] & 0xFFFFu) == 0)
                        v[8 * q + 2 * e] = 0.0f;
                    if ((w[e] & 0x80000000u) || (w[e] >> 16) == 0)
                        v[8 * q + 2 * e + 1] = 0.0f;
                }
            }
        }
        if (a.out_f32) {
            float4* o = reinterpret_cast<float4*>(
                static_cast<float*>(a.out) + pix * a.out_ps + a.out_coff + n);
#pragma unroll
            for (int q = 0; q < 4; q++)
                o[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2],
                                   v[4 * q + 3]);
        } else {
            uint4* o = reinterpret_cast<uint4*>(
                static_cast<__nv_bfloat16*>(a.out) + pix * a.out_ps +
                a.out_coff + n);
            o[0] = make_uint4(PackBf16(v[0], v[1]), PackBf16(v[2], v[3]),
                              PackBf16(v[4], v[5]), PackBf16(v[6], v[7]));
            o[1] = make_uint4(PackBf16(v[8], v[9]), PackBf16(v[10], v[11]),
                              PackBf16(v[12], v[13]), PackBf16(v[14], v[15]));
        }
    }

    FenceBeforeSync();
    __syncthreads();
    if (warp == 2) {
        FenceAfterSync();
        TmemFree(tmem, a.tmem_cols);
    }
}

__global__ void __launch_bounds__(kConvThreads, 1)
    WgradKernel(const __grid_constant__ CUtensorMap ta,
                const __grid_constant__ CUtensorMap tb, WgradArgs a) {
    constexpr uint32_t ATOM = 16384;   // 128 pixel rows x 64 channels
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = Align1024(smem_raw);
    const uint32_t stage_bytes = (2 + a.b_atoms) * ATOM;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + a.stages * stage_bytes);
    uint64_t* empty = full + a.stages;
    uint64_t* accum = empty + a.stages;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accum + 1);
    volatile int* cta_err = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ci_tiles = (a.cin + a.bn - 1) / a.bn;
    const int co_tiles = (a.cout + 127) / 128;
    int bx = blockIdx.x;
    const int ci_t = bx % ci_tiles;
    bx /= ci_tiles;
    const int co_t = bx % co_tiles;
    const int tap = bx / co_tiles;
    const int co0 = co_t * 128, ci0 = ci_t * a.bn;
    const int a_atoms = min(2, (a.cout - co0 + 63) / 64);
    const int b_atoms = min(a.b_atoms, (a.cin - ci0 + 63) / 64);
    const uint32_t tx = (uint32_t)(a_atoms + b_atoms) * ATOM;
    const int kb0 = blockIdx.y * a.kb_per_split;
    const int nk = min(a.kb_total, kb0 + a.kb_per_split) - kb0;
    if (nk <= 0) return;   // uniform over the CTA, before any allocation
    int dh, dw;
    TapOffset(a.taps, tap, dh, dw);

    if (threadIdx.x == 0) {
        for (int s = 0; s < a.stages; s++) {
            BarInit(&full[s], 1);
            BarInit(&empty[s], 1);
        }
        BarInit(accum, 1);
        *cta_err = 0;
        FenceBarrierInit();
        PrefetchTmap(&ta);
        PrefetchTmap(&tb);
    }
    if (warp == 2) TmemAlloc(tmem_slot, a.tmem_cols);
    FenceBeforeSync();
    __syncthreads();
    FenceAfterSync();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        int j = 0;
        for (; j < nk; j++) {
            const int s = j % a.stages;
            if (j >= a.stages &&
                !BarWait(&empty[s], ((j / a.stages) + 1) & 1, cta_err)) {
                Flag(cta_err, a.err);
                break;
            }
            const int g = kb0 + j;
            const int img = g / a.tiles_per_img;
            const int h0 = (g - img * a.tiles_per_img) * a.bh;
            uint8_t* sa = smem + s * stage_bytes;
            BarArriveExpectTx(&full[s], tx);
            for (int at = 0; at < a_atoms; at++)
                TmaLoad4D(sa + at * ATOM, &ta, &full[s], co0 + 64 * at, 0, h0,
                          img);
            for (int bt = 0; bt < b_atoms; bt++)
                TmaLoad4D(sa + (2 + bt) * ATOM, &tb, &full[s], ci0 + 64 * bt,
                          dw, h0 + dh, img);
        }
        for (int q = j > a.stages ? j - a.stages : 0; q < j; q++)
            if (!BarWaitDrain(&full[q % a.stages], (q / a.stages) & 1))
                Flag(cta_err, a.err);
    } else if (warp == 1 && lane == 0) {
        const uint32_t idesc = InstrDescBf16(kTileM, a.bn, true, true);
        const uint32_t base = SmemAddr(smem);
        for (int j = 0; j < nk; j++) {
            const int s = j % a.stages;
            if (!BarWait(&full[s], (j / a.stages) & 1, cta_err)) {
                Flag(cta_err, a.err);
                break;
            }
            FenceAfterSync();
            const uint32_t sa = base + s * stage_bytes;
            const uint32_t sb = sa + 2 * ATOM;
#pragma unroll
            for (int k = 0; k < 8; k++) {
                Mma(tmem, SmemDesc(sa + k * 2048, ATOM, 1024, 128),
                    SmemDesc(sb + k * 2048, ATOM, 1024, 128), idesc,
                    (j | k) != 0 ? 1u : 0u);
            }
            Commit(&empty[s]);
        }
        Commit(accum);
    }
    __syncwarp();

    const bool acc_ok = BarWaitDrain(accum, 0);
    FenceAfterSync();
    if (!acc_ok && threadIdx.x == 0) Flag(cta_err, a.err);
    const bool store = acc_ok && *cta_err == 0;
    const int co = co0 + warp * 32 + lane;
    for (int c = 0; c < a.bn; c += 16) {
        float v[16];
        TmemLoad16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
        if (!store || co >= a.cout) continue;
        float* d = a.dw + ((long long)co * a.taps + tap) * a.cin;
#pragma unroll
        for (int i = 0; i < 16; i++) {
            const int ci = ci0 + c + i;
            if (ci < a.cin) atomicAdd(d + ci, v[i]);
        }
    }

    FenceBeforeSync();
    __syncthreads();
    if (warp == 2) {
        FenceAfterSync();
        TmemFree(tmem, a.tmem_cols);
    }
}

__global__ void __launch_bounds__(kConvThreads, 1)
    WgradTKernel(const __grid_constant__ CUtensorMap tx,
                 const __grid_constant__ CUtensorMap tdy, WgradTArgs a) {
    constexpr uint32_t ATOM = 8192;   // 128 pixel rows x 32 channels
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = Align1024(smem_raw);
    const int b_atoms = a.bn / 32;
    const uint32_t stage_bytes = (4 + b_atoms) * ATOM;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + a.stages * stage_bytes);
    uint64_t* empty = full + a.stages;
    uint64_t* accum = empty + a.stages;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accum + 1);
    volatile int* cta_err = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // this CTA's M tile: atoms 4 blockIdx.x .. + 3 (atom = tap * ci_chunks
    // + chunk); the last tile may hold fewer
    const int atom0 = 4 * blockIdx.x;
    const int m_atoms = min(4, a.n_atoms - atom0);
    const uint32_t tx_bytes = (uint32_t)(m_atoms + b_atoms) * ATOM;
    const int kb0 = blockIdx.y * a.kb_per_split;
    const int nk = min(a.kb_total, kb0 + a.kb_per_split) - kb0;
    if (nk <= 0 || m_atoms <= 0) return;   // uniform, before any allocation

    if (threadIdx.x == 0) {
        for (int s = 0; s < a.stages; s++) {
            BarInit(&full[s], 1);
            BarInit(&empty[s], 1);
        }
        BarInit(accum, 1);
        *cta_err = 0;
        FenceBarrierInit();
        PrefetchTmap(&tx);
        PrefetchTmap(&tdy);
    }
    if (warp == 2) TmemAlloc(tmem_slot, a.tmem_cols);
    FenceBeforeSync();
    __syncthreads();
    FenceAfterSync();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        int j = 0;
        for (; j < nk; j++) {
            const int s = j % a.stages;
            if (j >= a.stages &&
                !BarWait(&empty[s], ((j / a.stages) + 1) & 1, cta_err)) {
                Flag(cta_err, a.err);
                break;
            }
            const int g = kb0 + j;
            const int img = g / a.tiles_per_img;
            const int h0 = (g - img * a.tiles_per_img) * a.bh;
            uint8_t* sa = smem + s * stage_bytes;
            BarArriveExpectTx(&full[s], tx_bytes);
            for (int m = 0; m < m_atoms; m++) {
                const int at = atom0 + m;
                const int tap = at / a.ci_chunks;
                const int chunk = at - tap * a.ci_chunks;
                int dh, dw;
                TapOffset(a.taps, tap, dh, dw);
                TmaLoad4D(sa + m * ATOM, &tx, &full[s], 32 * chunk, dw,
                          h0 + dh, img);
            }
            for (int bt = 0; bt < b_atoms; bt++)
                TmaLoad4D(sa + (4 + bt) * ATOM, &tdy, &full[s], 32 * bt, 0,
                          h0, img);
        }
        for (int q = j > a.stages ? j - a.stages : 0; q < j; q++)
            if (!BarWaitDrain(&full[q % a.stages], (q / a.stages) & 1))
                Flag(cta_err, a.err);
    } else if (warp == 1 && lane == 0) {
        const uint32_t idesc = InstrDescBf16(kTileM, a.bn, true, true);
        const uint32_t base = SmemAddr(smem);
        for (int j = 0; j < nk; j++) {
            const int s = j % a.stages;
            if (!BarWait(&full[s], (j / a.stages) & 1, cta_err)) {
                Flag(cta_err, a.err);
                break;
            }
            FenceAfterSync();
            const uint32_t sa = base + s * stage_bytes;
            const uint32_t sb = sa + 4 * ATOM;
            // MN-major, 64-byte swizzle: rows of 32 channels per pixel, 8-row
            // groups 512 B apart, atoms (32 M or N rows) 8 KiB apart; 16
            // pixels per MMA
#pragma unroll
            for (int k = 0; k < 8; k++) {
                Mma(tmem, SmemDesc(sa + k * 1024, ATOM, 512, 64),
                    SmemDesc(sb + k * 1024, ATOM, 512, 64), idesc,
                    (j | k) != 0 ? 1u : 0u);
            }
            Commit(&empty[s]);
        }
        Commit(accum);
    }
    __syncwarp();

    const bool acc_ok = BarWaitDrain(accum, 0);
    FenceAfterSync();
    if (!acc_ok && threadIdx.x == 0) Flag(cta_err, a.err);
    const bool store = acc_ok && *cta_err == 0;
    // TMEM lane = M row: atom (warp), channel lane of its chunk; columns are
    // output channels
    const int at = atom0 + warp;
    const int tap = at / a.ci_chunks;
    const int ci = 32 * (at - tap * a.ci_chunks) + lane;
    const bool row_ok = warp < m_atoms && ci < a.cin;
    for (int c = 0; c < a.bn; c += 16) {
        float v[16];
        TmemLoad16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
        if (!store || !row_ok) continue;
#pragma unroll
        for (int i = 0; i < 16; i++) {
            const int co = c + i;
            if (co < a.cout)
                atomicAdd(a.dw + ((long long)co * a.taps + tap) * a.cin + ci,
                          v[i]);
        }
    }

    FenceBeforeSync();
    __syncthreads();
    if (warp == 2) {
        FenceAfterSync();
        TmemFree(tmem, a.tmem_cols);
    }
}

}  // namespace nn
}  // namespace mplb

// ---------------------------------------------------------------------------
// Host side: tensor maps and launches.
// ---------------------------------------------------------------------------
#include <mutex>
#include <string>

#include "conv_host.h"

namespace mplb {
namespace nn {

namespace {

using tma::EncodeTiledFn;
using tma::Encoder;

bool CheckView(const View& v, const char* what, std::string& err) {
    char buf[256];
    const bool ok = v.ptr != nullptr && v.nimg > 0 && v.w > 0 && v.w <= 128 &&
                    128 % v.w == 0 && v.h > 0 && (v.h * v.w) % 128 == 0 &&
                    v.c > 0 && v.c % 16 == 0 && v.ps >= v.c && v.ps % 8 == 0 &&
                    reinterpret_cast<uintptr_t>(v.ptr) % 16 == 0;
    if (!ok) {
        snprintf(buf, sizeof buf,
                 "%s view unsupported (nimg %d, h %d, w %d, c %d, ps %lld)",
                 what, v.nimg, v.h, v.w, v.c, v.ps);
        err = buf;
    }
    return ok;
}

bool EncodeAct(CUtensorMap* m, const View& v, int box_c, int swizzle,
               std::string& err) {
    EncodeTiledFn enc = Encoder();
    if (enc == nullptr) {
        err = "cuTensorMapEncodeTiled is not available";
        return false;
    }
    const cuuint64_t dims[4] = {(cuuint64_t)v.c, (cuuint64_t)v.w,
                                (cuuint64_t)v.h, (cuuint64_t)v.nimg};
    const cuuint64_t strides[3] = {(cuuint64_t)v.ps * 2,
                                   (cuuint64_t)v.ps * 2 * v.w,
                                   (cuuint64_t)v.ps * 2 * v.w * v.h};
    const cuuint32_t box[4] = {(cuuint32_t)box_c, (cuuint32_t)v.w,
                               (cuuint32_t)(128 / v.w), 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = enc(
        m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, v.ptr, dims, strides, box,
        estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
        swizzle == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        err = "tensor map of an activation view rejected (CUresult " +
              std::to_string((int)r) + ")";
        return false;
    }
    return true;
}

bool EncodeRows(CUtensorMap* m, const void* ptr, int rows, int kdim,
                int box_k, int box_rows, int swizzle, std::string& err) {
    EncodeTiledFn enc = Encoder();
    if (enc == nullptr) {
        err = "cuTensorMapEncodeTiled is not available";
        return false;
    }
    if (reinterpret_cast<uintptr_t>(ptr) % 16 != 0 || kdim % 8 != 0) {
        err = "weight matrix misaligned";
        return false;
    }
    const cuuint64_t dims[2] = {(cuuint64_t)kdim, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)kdim * 2};
    const cuuint32_t box[2] = {(cuuint32_t)box_k, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = enc(
        m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims,
        strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
        swizzle == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        err = "tensor map of a weight matrix rejected (CUresult " +
              std::to_string((int)r) + ")";
        return false;
    }
    return true;
}

int Pow2Cols(int n) {
    int c = 32;
    while (c < n) c *= 2;
    return c;
}

// Largest divisor of c that is a multiple of 16 and at most 256.
int PickBn(int c) {
    for (int bn = 256; bn >= 16; bn -= 16)
        if (c % bn == 0) return bn;
    return 0;
}

constexpr int kSmemPerSm = 228 * 1024;
constexpr int kSmemMax = 227 * 1024;

// Dynamic shared memory for a launch: pads the request so that the CTAs an
// SM can hold never ask for more than its 512 TMEM columns together.
int ResidencySafeSmem(int smem, int tmem_cols) {
    const int max_ctas = 512 / tmem_cols;
    const int floor_bytes = kSmemPerSm / max_ctas - 1024;
    if (smem < floor_bytes) smem = floor_bytes;
    return smem > kSmemMax ? kSmemMax : smem;
}

template <int BK>
cudaError_t SetSmemAttr() {
    static cudaError_t e = cudaFuncSetAttribute(
        ConvKernel<BK>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemMax);
    return e;
}

cudaError_t SetWgradTSmemAttr() {
    static cudaError_t e = cudaFuncSetAttribute(
        WgradTKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemMax);
    return e;
}

cudaError_t SetWgradSmemAttr() {
    static cudaError_t e = cudaFuncSetAttribute(
        WgradKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemMax);
    return e;
}

}  // namespace

bool LaunchConv(const View& x, const void* w, int taps, const float* bias,
                int relu, const View& y, bool y_f32, const View* mask,
                cudaStream_t stream, int* err_dev, std::string& err) {
    if (!CheckView(x, "input", err) || !CheckView(y, "output", err))
        return false;
    if (mask != nullptr && !CheckView(*mask, "mask", err)) return false;
    if ((taps != 9 && taps != 1) || w == nullptr ||
        x.nimg != y.nimg || x.h != y.h || x.w != y.w ||
        (mask != nullptr &&
         (mask->nimg != y.nimg || mask->h != y.h || mask->w != y.w ||
          mask->c < y.c))) {
        err = "convolution shapes do not match";
        return false;
    }
    if (y_f32 && (y.ps % 4 != 0)) {
        err = "fp32 output pixel stride must be a multiple of 4";
        return false;
    }
    const int bk = x.c % 64 == 0 ? 64 : 32;
    const int bn = PickBn(y.c);
    if (bn == 0) {
        err = "output channels must be a multiple of 16";
        return false;
    }
    CUtensorMap ta, tb;
    if (!EncodeAct(&ta, x, bk, bk * 2, err)) return false;
    if (!EncodeRows(&tb, w, y.c, taps * x.c, bk, bn, bk * 2, err)) return false;
    ConvArgs a{};
    a.H = x.h;
    a.W = x.w;
    a.tiles_per_img = x.h * x.w / kTileM;
    a.bh = kTileM / x.w;
    a.cin = x.c;
    a.taps = taps;
    a.nkb = taps * ((x.c + bk - 1) / bk);
    a.cout = y.c;
    a.bn = bn;
    a.stages = 4;
    while (a.stages > 2 && ConvSmemBytes(bk, bn, a.stages) > 200 * 1024)
        a.stages--;
    a.tmem_cols = Pow2Cols(bn);
    a.out = y.ptr;
    a.out_ps = y.ps;
    a.out_coff = 0;
    a.out_f32 = y_f32 ? 1 : 0;
    a.bias = bias;
    a.relu = relu;
    a.mask = mask ? static_cast<const __nv_bfloat16*>(mask->ptr) : nullptr;
    a.mask_ps = mask ? mask->ps : 0;
    a.mask_coff = 0;
    a.err = err_dev;
    const int smem = ResidencySafeSmem(ConvSmemBytes(bk, bn, a.stages),
                                       a.tmem_cols);
    const dim3 grid(x.nimg * a.tiles_per_img, y.c / bn);
    cudaError_t e;
    if (bk == 64) {
        e = SetSmemAttr<64>();
        if (e == cudaSuccess)
            ConvKernel<64><<<grid, kConvThreads, smem, stream>>>(ta, tb, a);
    } else {
        e = SetSmemAttr<32>();
        if (e == cudaSuccess)
            ConvKernel<32><<<grid, kConvThreads, smem, stream>>>(ta, tb, a);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        err = std::string("convolution launch: ") + cudaGetErrorString(e);
        return false;
    }
    return true;
}

bool LaunchWgrad(const View& dy, const View& x, int taps, float* dw,
                 int sm_count, cudaStream_t stream, int* err_dev,
                 std::string& err) {
    if (!CheckView(dy, "output gradient", err) || !CheckView(x, "input", err))
        return false;
    if ((taps != 9 && taps != 1) || dw == nullptr || x.nimg != dy.nimg ||
        x.h != dy.h || x.w != dy.w) {
        err = "weight-gradient shapes do not match";
        return false;
    }
    if (dy.c <= 64) {
        // few output channels: taps x input channels along M (WgradTKernel)
        CUtensorMap tx, tdy;
        if (!EncodeAct(&tx, x, 32, 64, err) || !EncodeAct(&tdy, dy, 32, 64, err))
            return false;
        WgradTArgs t{};
        t.H = x.h;
        t.W = x.w;
        t.tiles_per_img = x.h * x.w / kTileM;
        t.bh = kTileM / x.w;
        t.taps = taps;
        t.cout = dy.c;
        t.cin = x.c;
        t.ci_chunks = (x.c + 31) / 32;
        t.n_atoms = taps * t.ci_chunks;
        t.bn = 32 * ((dy.c + 31) / 32);
        t.stages = 4;
        t.tmem_cols = Pow2Cols(t.bn);
        t.kb_total = x.nimg * t.tiles_per_img;
        const int mtiles = (t.n_atoms + 3) / 4;
        int splits = (2 * sm_count + mtiles - 1) / mtiles;
        if (splits < 1) splits = 1;
        if (splits > t.kb_total) splits = t.kb_total;
        t.kb_per_split = (t.kb_total + splits - 1) / splits;
        splits = (t.kb_total + t.kb_per_split - 1) / t.kb_per_split;
        t.dw = dw;
        t.err = err_dev;
        const int smem = ResidencySafeSmem(WgradTSmemBytes(t.bn, t.stages),
                                           t.tmem_cols);
        cudaError_t e = SetWgradTSmemAttr();
        if (e == cudaSuccess)
            WgradTKernel<<<dim3(mtiles, splits), kConvThreads, smem, stream>>>(
                tx, tdy, t);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e != cudaSuccess) {
            err = std::string("weight-gradient launch: ") +
                  cudaGetErrorString(e);
            return false;
        }
        return true;
    }
    CUtensorMap ta, tb;
    if (!EncodeAct(&ta, dy, 64, 128, err) || !EncodeAct(&tb, x, 64, 128, err))
        return false;
    WgradArgs a{};
    a.H = x.h;
    a.W = x.w;
    a.tiles_per_img = x.h * x.w / kTileM;
    a.bh = kTileM / x.w;
    a.taps = taps;
    a.cout = dy.c;
    a.cin = x.c;
    a.b_atoms = (x.c + 63) / 64;
    if (a.b_atoms > 4) a.b_atoms = 4;
    a.bn = 64 * a.b_atoms;
    a.stages = a.b_atoms >= 3 ? 2 : (a.b_atoms == 2 ? 3 : 4);
    a.tmem_cols = Pow2Cols(a.bn);
    a.kb_total = x.nimg * a.tiles_per_img;
    const int blocks = taps * ((dy.c + 127) / 128) * ((x.c + a.bn - 1) / a.bn);
    int splits = (2 * sm_count + blocks - 1) / blocks;
    if (splits < 1) splits = 1;
    if (splits > a.kb_total) splits = a.kb_total;
    a.kb_per_split = (a.kb_total + splits - 1) / splits;
    splits = (a.kb_total + a.kb_per_split - 1) / a.kb_per_split;
    a.dw = dw;
    a.err = err_dev;
    const int smem = ResidencySafeSmem(WgradSmemBytes(a.b_atoms, a.stages),
                                       a.tmem_cols);
    cudaError_t e = SetWgradSmemAttr();
    if (e == cudaSuccess)
        WgradKernel<<<dim3(blocks, splits), kConvThreads, smem, stream>>>(
            ta, tb, a);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        err = std::string("weight-gradient launch: ") + cudaGetErrorString(e);
        return false;
    }
    return true;
}

}  // namespace nn
}  // namespace mplb
