// conv_tma.cu -- the proposal network's 3^3 convolutions as implicit GEMMs on the sm_100a
// tensor cores with TMA-fed operands: k_conv_tma for 32-channel grids onto 4^3 output grids
// (optionally with the 1^3 head fused into its epilogue), k_conv8_tma for the first layer
// (8 padded channels, 8^3 -> 6^3; described above the kernel).
//
// k_conv_tma.  Rows are (window, x, y, z) of the output grid, 64 per window; a block
// computes the 128 rows of two windows for all N output channels.  K runs over the 27 kernel
// offsets (dx, dy, dz) x 32 channels.  For offset t the 128 x 32 A tile is one box of the 5-D tensor
// (channel, z, y, x, window) of the input: channels 0..31, z, y, x from offset - pad over 4
// cells each, windows w0, w0 + 1.  One tiled TMA copy moves it into shared memory with the
// 64-byte swizzle (each 64-byte row holds the 32 channels of one output row), and coordinates
// outside the grid (the "same" padding, a missing second window) read as zeros.  The N x 32
// slice of the weights (row pitch ldb, columns 32 t .. 32 t + 31) is a second tiled copy.
// Both land in one stage of a six-stage ring; one thread issues the copies, waits for a
// stage's transaction count, issues the two K = 16 MMAs of the offset (the second starting
// 32 bytes into the swizzled rows) and commits them to the stage's "empty" barrier, which
// releases the stage for the copies of offset t + 6.  The epilogue is the one of the
// register-staged GEMM (gemm_umma.cu): bias, optional GELU, FP32 and/or BF16 rows, and, when
// asked, the head's four outputs per row from the BF16-rounded channels.
//
// The accumulation order (offset by offset, K = 16 steps in K order) is the register-staged
// kernel's, so both produce identical sums.  Every mbarrier wait is bounded; after a wait
// that gives up the kernel drains the copies it issued (bounded), sets kStatTimeout and skips
// the epilogue.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <atomic>

#include "internal.h"
#include "learned.h"
#include "umma.cuh"

namespace isg {
namespace {

constexpr int kCtThreads = 128;
constexpr int kCtStages = 6;
constexpr int kCtTaps = 27;
constexpr uint32_t kCtA = 128u * 64u;         // A tile bytes: 128 rows x 32 BF16
constexpr uint32_t kCtWaitPolls = 1u << 22;

struct ConvTmaArgs {
    int M, N, pad;
    const float* bias;
    float* C;
    int ldc, accumulate;
    __nv_bfloat16* O;
    int ldo, gelu;
    int* status;
    uint32_t tmem_cols, b_stage;   // B bytes per stage, rounded up to 1024
    const float* head_w;           // optional fused 1^3 head: head_w[4][N], head_b[4]
    const float* head_b;
    float* head_out;               // [M][4]
};

// K-major operand in the 64-byte swizzle layout: 64-byte rows, 8-row groups 512 bytes apart
// (SBO), leading offset field 1 as for every swizzled K-major layout, layout type 4.
__device__ __forceinline__ uint64_t umma_desc_sw64(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(512u >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)4 << 61);
}

__device__ __forceinline__ void ct_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, int c4,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int c0, int c1, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ float ct_gelu(float x) {
    const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
    return 0.5f * x * (1.f + tanhf(u));
}

__global__ void __launch_bounds__(kCtThreads) k_conv_tma(const __grid_constant__ CUtensorMap tA,
                                                         const __grid_constant__ CUtensorMap tB,
                                                         const ConvTmaArgs g) {
    extern __shared__ unsigned char smem_raw[];
    // stages start on 1024-byte boundaries (the swizzle pattern repeats every 512 bytes)
    unsigned char* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    const uint32_t stage_bytes = kCtA + g.b_stage;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + kCtStages * stage_bytes);
    uint64_t* empty = full + kCtStages;
    uint64_t* done = empty + kCtStages;
    uint32_t* slot = reinterpret_cast<uint32_t*>(done + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int N = g.N;

    if (warp == 0) tmem_alloc(slot, g.tmem_cols);
    if (tid == 0) {
        for (int s = 0; s < kCtStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        mbar_init_fence();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t taddr = *slot;

    bool ok = true;
    if (tid == 0) {
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tA)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tB)) : "memory");
        const int w0 = 2 * (int)blockIdx.x;
        const uint32_t tx = kCtA + (uint32_t)N * 64u;
        const uint32_t idesc = umma_idesc_bf16(128, N);
        auto issue = [&](int t) {
            const int s = t % kCtStages;
            unsigned char* sA = smem + s * stage_bytes;
            const int dx = t / 9, dy = (t / 3) % 3, dz = t % 3;
            ct_expect_tx(&full[s], tx);
            tma_load_5d(sA, &tA, 0, dz - g.pad, dy - g.pad, dx - g.pad, w0, &full[s]);
            tma_load_2d(sA + kCtA, &tB, 32 * t, 0, &full[s]);
        };
        int issued = 0;
        for (; issued < kCtStages && issued < kCtTaps; ++issued) issue(issued);
        int t = 0;
        for (; t < kCtTaps && ok; ++t) {
            const int s = t % kCtStages;
            ok = mbar_wait(&full[s], (uint32_t)((t / kCtStages) & 1), kCtWaitPolls);
            if (!ok) break;
            tc_fence_after();
            const uint32_t a0 = smem_u32(smem + s * stage_bytes), b0 = a0 + kCtA;
#pragma unroll
            for (int j = 0; j < 2; ++j)
                umma_bf16(taddr, umma_desc_sw64(a0 + 32u * j), umma_desc_sw64(b0 + 32u * j), idesc,
                          (t > 0 || j > 0) ? 1u : 0u);
            umma_commit(&empty[s]);
            // the stage of offset t-1 takes offset t-1+S once offset t-1's MMAs are done
            if (t >= 1 && issued < kCtTaps) {
                const int ps = (t - 1) % kCtStages;
                ok = mbar_wait(&empty[ps], (uint32_t)(((t - 1) / kCtStages) & 1), kCtWaitPolls);
                if (ok) issue(issued++);
            }
        }
        if (!ok) {
            // copies issued for offsets t .. issued-1 may still be in flight: let them land
            for (int u = t; u < issued; ++u) mbar_wait(&full[u % kCtStages], (uint32_t)((u / kCtStages) & 1), 1u << 20);
            atomicOr(g.status, kStatTimeout);
        }
        umma_commit(done);   // arrives once every MMA issued above has completed
    }
    ok = __syncthreads_and(ok);
    const bool fin = mbar_wait(done, 0u, kCtWaitPolls);
    tc_fence_after();
    if (!fin && tid == 0) atomicOr(g.status, kStatTimeout);
    if (ok && fin) {
        // warp w reads TMEM lanes 32 w .. 32 w + 31: one output row per thread
        const int row = (int)blockIdx.x * 128 + warp * 32 + lane;
        float hacc[4] = {0.f, 0.f, 0.f, 0.f};
        if (g.head_out)
            for (int o = 0; o < 4; ++o) hacc[o] = g.head_b[o];
        for (int cb = 0; cb < N; cb += 16) {
            float v[16];
            tmem_ld16(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)cb, v);
            if (row < g.M) {
#pragma unroll
                for (int i = 0; i < 16; ++i) v[i] += g.bias ? g.bias[cb + i] : 0.f;
                if (g.C) {
                    float4* cp = reinterpret_cast<float4*>(g.C + (size_t)row * g.ldc + cb);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        float4 x = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
                        if (g.accumulate) {
                            const float4 o = cp[q];
                            x.x += o.x; x.y += o.y; x.z += o.z; x.w += o.w;
                        }
                        cp[q] = x;
                    }
                }
                if (g.O || g.head_out) {
#pragma unroll
                    for (int q = 0; q < 2; ++q) {
                        uint32_t w[4];
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const float a = g.gelu ? ct_gelu(v[8 * q + 2 * e]) : v[8 * q + 2 * e];
                            const float b = g.gelu ? ct_gelu(v[8 * q + 2 * e + 1]) : v[8 * q + 2 * e + 1];
                            const __nv_bfloat162 h2 = __floats2bfloat162_rn(a, b);
                            w[e] = *reinterpret_cast<const uint32_t*>(&h2);
                            if (g.head_out) {   // the head reads the BF16-rounded channels, in order
                                const int c = cb + 8 * q + 2 * e;
                                const float ha = __low2float(h2), hb = __high2float(h2);
#pragma unroll
                                for (int o = 0; o < 4; ++o) hacc[o] = fmaf(ha, g.head_w[o * N + c], hacc[o]);
#pragma unroll
                                for (int o = 0; o < 4; ++o) hacc[o] = fmaf(hb, g.head_w[o * N + c + 1], hacc[o]);
                            }
                        }
                        if (g.O)
                            reinterpret_cast<uint4*>(g.O + (size_t)row * g.ldo + cb)[q] = make_uint4(w[0], w[1], w[2], w[3]);
                    }
                }
            }
        }
        if (g.head_out && row < g.M)
            *reinterpret_cast<float4*>(g.head_out + (size_t)row * 4) = make_float4(hacc[0], hacc[1], hacc[2], hacc[3]);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(taddr, g.tmem_cols);
}

// First layer: 3^3 convolution over an 8-channel grid (8^3 cells) onto its 6^3 valid output
// cells.  A block computes two windows: each window's 216 rows sit in a 256-row tile covered
// by two M = 128 MMAs, the four accumulators N TMEM columns apart, and the two windows share
// each step's weight slices.  Kernel offset t is one
// 216 x 8 box (16-byte rows, no swizzle) copied densely into a 256-row buffer, which is the
// canonical no-swizzle K-major layout with 8-row groups 128 bytes apart; the two offsets of
// a K = 16 step sit in consecutive buffers (leading offset 4 KB), as do their N x 8 weight
// slices.  Offset 27 pads K to 224: its box lies wholly outside the tensor (window index
// nwin) and TMA fills it with zeros.  Rows 216..255 of a buffer are never written and feed
// only the discarded accumulator rows.
constexpr int kC8Stages = 4;
constexpr int kC8Win = 2;                     // windows per block
constexpr int kC8Pairs = 14;                  // 28 offsets (27 + the zero pad), two per K step
constexpr uint32_t kC8TapA = 256u * 16u;      // 256 rows x 8 BF16

struct Conv8Args {
    int M, N, nwin;
    const float* bias;
    float* C;
    int ldc, accumulate;
    __nv_bfloat16* O;
    int ldo, gelu;
    int* status;
    uint32_t tmem_cols;
};

__global__ void __launch_bounds__(kCtThreads) k_conv8_tma(const __grid_constant__ CUtensorMap tA,
                                                          const __grid_constant__ CUtensorMap tB,
                                                          const Conv8Args g) {
    extern __shared__ unsigned char smem_raw[];
    unsigned char* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    const int N = g.N;
    const uint32_t tapB = (uint32_t)N * 16u;
    const uint32_t stage_bytes = kC8Win * 2u * kC8TapA + 2u * tapB;   // [window][offset] A, then B
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + kC8Stages * stage_bytes);
    uint64_t* empty = full + kC8Stages;
    uint64_t* done = empty + kC8Stages;
    uint32_t* slot = reinterpret_cast<uint32_t*>(done + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int win0 = kC8Win * (int)blockIdx.x;

    if (warp == 0) tmem_alloc(slot, g.tmem_cols);
    if (tid == 0) {
        for (int s = 0; s < kC8Stages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        mbar_init_fence();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t taddr = *slot;

    bool ok = true;
    if (tid == 0) {
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tA)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tB)) : "memory");
        const uint32_t tx = kC8Win * 2u * 216u * 16u + 2u * tapB;
        const uint32_t idesc = umma_idesc_bf16(128, N);
        auto issue = [&](int p) {
            const int s = p % kC8Stages;
            unsigned char* st = smem + s * stage_bytes;
            ct_expect_tx(&full[s], tx);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int t = 2 * p + h;
                // a window index at or past nwin (a block's missing second window, or the pad
                // offset) lies outside the tensor and reads as zeros
#pragma unroll
                for (int w = 0; w < kC8Win; ++w) {
                    unsigned char* dst = st + (uint32_t)(2 * w + h) * kC8TapA;
                    if (t < kCtTaps) tma_load_5d(dst, &tA, 0, t % 3, (t / 3) % 3, t / 9, win0 + w, &full[s]);
                    else tma_load_5d(dst, &tA, 0, 0, 0, 0, g.nwin, &full[s]);
                }
                tma_load_2d(st + kC8Win * 2u * kC8TapA + h * tapB, &tB, 8 * t, 0, &full[s]);
            }
        };
        int issued = 0;
        for (; issued < kC8Stages && issued < kC8Pairs; ++issued) issue(issued);
        int p = 0;
        for (; p < kC8Pairs && ok; ++p) {
            const int s = p % kC8Stages;
            ok = mbar_wait(&full[s], (uint32_t)((p / kC8Stages) & 1), kCtWaitPolls);
            if (!ok) break;
            tc_fence_after();
            const uint32_t a0 = smem_u32(smem + s * stage_bytes), b0 = a0 + kC8Win * 2u * kC8TapA;
            const uint64_t bd = umma_smem_desc(b0, tapB, 128u);
#pragma unroll
            for (int w = 0; w < kC8Win; ++w)
#pragma unroll
                for (int h = 0; h < 2; ++h)
                    umma_bf16(taddr + (uint32_t)((2 * w + h) * N),
                              umma_smem_desc(a0 + (uint32_t)(2 * w) * kC8TapA + (uint32_t)h * 2048u, kC8TapA, 128u), bd,
                              idesc, p > 0 ? 1u : 0u);
            umma_commit(&empty[s]);
            if (p >= 1 && issued < kC8Pairs) {
                const int ps = (p - 1) % kC8Stages;
                ok = mbar_wait(&empty[ps], (uint32_t)(((p - 1) / kC8Stages) & 1), kCtWaitPolls);
                if (ok) issue(issued++);
            }
        }
        if (!ok) {
            for (int u = p; u < issued; ++u) mbar_wait(&full[u % kC8Stages], (uint32_t)((u / kC8Stages) & 1), 1u << 20);
            atomicOr(g.status, kStatTimeout);
        }
        umma_commit(done);
    }
    ok = __syncthreads_and(ok);
    const bool fin = mbar_wait(done, 0u, kCtWaitPolls);
    tc_fence_after();
    if (!fin && tid == 0) atomicOr(g.status, kStatTimeout);
    if (ok && fin) {
        for (int wh = 0; wh < 2 * kC8Win; ++wh) {
            const int u = (wh & 1) * 128 + warp * 32 + lane;     // output cell of window win0 + wh / 2
            const int row = (win0 + (wh >> 1)) * 216 + u;
            for (int cb = 0; cb < N; cb += 16) {
                float v[16];
                tmem_ld16(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)(wh * N + cb), v);
                if (u < 216 && row < g.M) {
#pragma unroll
                    for (int i = 0; i < 16; ++i) v[i] += g.bias ? g.bias[cb + i] : 0.f;
                    if (g.C) {
                        float4* cp = reinterpret_cast<float4*>(g.C + (size_t)row * g.ldc + cb);
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            float4 x = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
                            if (g.accumulate) {
                                const float4 o = cp[q];
                                x.x += o.x; x.y += o.y; x.z += o.z; x.w += o.w;
                            }
                            cp[q] = x;
                        }
                    }
                    if (g.O) {
                        uint4* op = reinterpret_cast<uint4*>(g.O + (size_t)row * g.ldo + cb);
#pragma unroll
                        for (int q = 0; q < 2; ++q) {
                            uint32_t w[4];
#pragma unroll
                            for (int e = 0; e < 4; ++e) {
                                const float a = g.gelu ? ct_gelu(v[8 * q + 2 * e]) : v[8 * q + 2 * e];
                                const float b = g.gelu ? ct_gelu(v[8 * q + 2 * e + 1]) : v[8 * q + 2 * e + 1];
                                const __nv_bfloat162 h2 = __floats2bfloat162_rn(a, b);
                                w[e] = *reinterpret_cast<const uint32_t*>(&h2);
                            }
                            op[q] = make_uint4(w[0], w[1], w[2], w[3]);
                        }
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(taddr, g.tmem_cols);
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(tensor_map_encoder());
}

bool conv8_shape(const GemmArgs& g) {
    return g.conv_in && g.conv_C == 8 && g.conv_Gi == 8 && g.conv_Go == 6 && g.conv_pad == 0 && g.K == 224 &&
           g.M % 216 == 0 && g.N % 16 == 0 && g.N <= 64;
}

bool conv32_shape(const GemmArgs& g) {
    return g.conv_in && g.conv_C == 32 && g.conv_Go == 4 && g.K == 27 * 32 && (g.conv_pad == 0 || g.conv_pad == 1) &&
           g.conv_Gi == 4 + 2 - 2 * g.conv_pad && g.M % 64 == 0 && g.N % 16 == 0 && g.N <= 256;
}

int launch_conv8_tma(const GemmArgs& g, cudaStream_t s) {
    // tensor-map rules checked before any copy: 16-byte aligned bases, strides multiples of
    // 16 bytes, 16-byte inner boxes, innermost coordinates 0 and 8 t (16 t bytes)
    if ((reinterpret_cast<uintptr_t>(g.conv_in) & 15) || (reinterpret_cast<uintptr_t>(g.B) & 15) || g.ldb % 8 ||
        g.ldb < g.K)
        return fail(ISING_ERR_ARG, "TMA convolution: operands must be 16-byte aligned with ldb % 8 == 0");
    const int nwin = g.M / 216;
    PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
    CUtensorMap tA, tB;
    {
        const cuuint64_t dims[5] = {8, 8, 8, 8, (cuuint64_t)nwin};
        const cuuint64_t strides[4] = {16, 128, 1024, 8192};
        const cuuint32_t box[5] = {8, 6, 6, 6, 1};
        const cuuint32_t es[5] = {1, 1, 1, 1, 1};
        if (enc(&tA, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<__nv_bfloat16*>(g.conv_in), dims, strides, box, es,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return fail(ISING_ERR_CUDA, "cuTensorMapEncodeTiled (first-layer windows) failed");
    }
    {
        const cuuint64_t dims[2] = {(cuuint64_t)g.K, (cuuint64_t)g.N};
        const cuuint64_t strides[1] = {(cuuint64_t)g.ldb * 2};
        const cuuint32_t box[2] = {8, (cuuint32_t)g.N};
        const cuuint32_t es[2] = {1, 1};
        if (enc(&tB, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(g.B), dims, strides, box, es,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return fail(ISING_ERR_CUDA, "cuTensorMapEncodeTiled (first-layer weights) failed");
    }
    Conv8Args a{};
    a.M = g.M; a.N = g.N; a.nwin = nwin; a.bias = g.bias; a.C = g.C; a.ldc = g.ldc; a.accumulate = g.accumulate;
    a.O = g.O; a.ldo = g.ldo; a.gelu = g.gelu; a.status = g.status;
    const int cols = kC8Win * 2 * g.N;   // two 128-row halves per window
    a.tmem_cols = cols <= 32 ? 32 : cols <= 64 ? 64 : cols <= 128 ? 128 : 256;
    int smem = 1024 + kC8Stages * (int)(kC8Win * 2u * kC8TapA + 2u * (uint32_t)g.N * 16u) + (2 * kC8Stages + 1) * 8 + 16;
    // the shared-memory limit is a per-device attribute of the kernel: raise it once per device
    static std::atomic<unsigned long long> attr_set{0};
    {
        int dev = 0;
        ISG_CUDA(cudaGetDevice(&dev));
        const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
        if (!bit || !(attr_set.load() & bit)) {
            ISG_CUDA(cudaFuncSetAttribute(k_conv8_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
            attr_set.fetch_or(bit);
        }
    }
    for (;;) {
        int occ = 0;
        ISG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_conv8_tma, kCtThreads, smem));
        if (occ * (int)a.tmem_cols <= 512 || smem >= 200 * 1024) break;
        smem += 8 * 1024;
    }
    k_conv8_tma<<<(nwin + kC8Win - 1) / kC8Win, kCtThreads, smem, s>>>(tA, tB, a);
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}

}  // namespace

// the driver's tensor-map encoder, looked up once (thread-safe static initialisation)
void* tensor_map_encoder() {
    static void* const fn = []() -> void* {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return p;
        return nullptr;
    }();
    return fn;
}

bool conv_tma_applies(const GemmArgs& g) {
    return (conv32_shape(g) || conv8_shape(g)) && encode_fn() != nullptr;
}

int launch_conv_tma(const GemmArgs& g, cudaStream_t s) {
    if (!conv_tma_applies(g)) return fail(ISING_ERR_ARG, "TMA convolution: unsupported shape");
    if (g.C && (g.ldc % 4 || g.ldc < g.N || (reinterpret_cast<uintptr_t>(g.C) & 15)))
        return fail(ISING_ERR_ARG, "GEMM FP32 output needs a 16-byte aligned base and ldc % 4 == 0");
    if (g.O && (g.ldo % 8 || g.ldo < g.N || (reinterpret_cast<uintptr_t>(g.O) & 15)))
        return fail(ISING_ERR_ARG, "GEMM BF16 output needs a 16-byte aligned base and ldo % 8 == 0");
    if (g.head_out && ((reinterpret_cast<uintptr_t>(g.head_out) & 15) || !g.head_w || !g.head_b || conv8_shape(g)))
        return fail(ISING_ERR_ARG, "fused head: 16-byte aligned output, weights and bias, 32-channel layers only");
    if (conv8_shape(g)) return launch_conv8_tma(g, s);
    // the tensor-map rules, checked before any copy is issued: 16-byte aligned bases, strides
    // multiples of 16 bytes, a 64-byte inner box (<= the 64-byte swizzle span), boxes <= 256
    if ((reinterpret_cast<uintptr_t>(g.conv_in) & 15) || (reinterpret_cast<uintptr_t>(g.B) & 15) || g.ldb % 8 ||
        g.ldb < g.K)
        return fail(ISING_ERR_ARG, "TMA convolution: operands must be 16-byte aligned with ldb % 8 == 0");
    const int nwin = g.M / 64, Gi = g.conv_Gi;
    PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
    CUtensorMap tA, tB;
    {
        const cuuint64_t dims[5] = {32, (cuuint64_t)Gi, (cuuint64_t)Gi, (cuuint64_t)Gi, (cuuint64_t)nwin};
        const cuuint64_t strides[4] = {64, (cuuint64_t)Gi * 64, (cuuint64_t)Gi * Gi * 64, (cuuint64_t)Gi * Gi * Gi * 64};
        const cuuint32_t box[5] = {32, 4, 4, 4, 2};
        const cuuint32_t es[5] = {1, 1, 1, 1, 1};
        if (enc(&tA, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<__nv_bfloat16*>(g.conv_in), dims, strides, box, es,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return fail(ISING_ERR_CUDA, "cuTensorMapEncodeTiled (activations) failed");
    }
    {
        const cuuint64_t dims[2] = {(cuuint64_t)g.K, (cuuint64_t)g.N};
        const cuuint64_t strides[1] = {(cuuint64_t)g.ldb * 2};
        const cuuint32_t box[2] = {32, (cuuint32_t)g.N};
        const cuuint32_t es[2] = {1, 1};
        if (enc(&tB, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(g.B), dims, strides, box, es,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return fail(ISING_ERR_CUDA, "cuTensorMapEncodeTiled (weights) failed");
    }
    ConvTmaArgs a{};
    a.M = g.M; a.N = g.N; a.pad = g.conv_pad; a.bias = g.bias; a.C = g.C; a.ldc = g.ldc; a.accumulate = g.accumulate;
    a.O = g.O; a.ldo = g.ldo; a.gelu = g.gelu; a.status = g.status;
    a.tmem_cols = g.N <= 32 ? 32 : g.N <= 64 ? 64 : g.N <= 128 ? 128 : 256;
    a.head_w = g.head_w; a.head_b = g.head_b; a.head_out = g.head_out;
    a.b_stage = ((uint32_t)g.N * 64u + 1023u) & ~1023u;
    int smem = 1024 + kCtStages * (int)(kCtA + a.b_stage) + (2 * kCtStages + 1) * 8 + 16;
    // the shared-memory limit is a per-device attribute of the kernel: raise it once per device
    static std::atomic<unsigned long long> attr_set{0};
    {
        int dev = 0;
        ISG_CUDA(cudaGetDevice(&dev));
        const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
        if (!bit || !(attr_set.load() & bit)) {
            ISG_CUDA(cudaFuncSetAttribute(k_conv_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
            attr_set.fetch_or(bit);
        }
    }
    if (smem > 200 * 1024) return fail(ISING_ERR_ARG, "TMA convolution: N too large for the stage ring");
    // resident blocks x TMEM columns must fit the SM's 512 columns
    for (;;) {
        int occ = 0;
        ISG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_conv_tma, kCtThreads, smem));
        if (occ * (int)a.tmem_cols <= 512 || smem >= 200 * 1024) break;
        smem += 8 * 1024;
    }
    k_conv_tma<<<(nwin + 1) / 2, kCtThreads, smem, s>>>(tA, tB, a);
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}

}  // namespace isg
