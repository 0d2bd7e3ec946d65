// gemm_umma.cu -- C = A * B^T on the sm_100a tensor cores (tcgen05.mma kind::f16, BF16 in,
// FP32 accumulation in TMEM), the matrix engine of the learned patch proposal: every
// convolution of its forward and backward passes is an im2col matrix times a weight matrix.
//
// A is M x K, B is N x K, both BF16 with K contiguous (row pitches lda, ldb, multiples of
// 8 elements), K a multiple of 16, N a multiple of 16 up to 256; A holds ceil(M/128)*128
// readable rows.  For a 32-channel 3^3 convolution A is not stored: the loader gathers its
// 16-byte pieces from the channel-last input grid (implicit GEMM), zero outside the grid.  One block of 128 threads computes a 128-row tile for all N columns:
// chunks of 64 values of K are staged by all threads into a two-stage ring in the canonical
// no-swizzle layout (umma.cuh), thread 0 issues the MMAs and commits them to the stage's
// mbarrier, and the block refills a stage once that mbarrier reports its MMAs done.  The
// epilogue reads each thread's TMEM lane (one output row), adds the bias, applies GELU when
// asked, and stores FP32 and/or BF16 rows.  Every mbarrier wait is bounded; a wait that
// gives up sets kStatTimeout and skips the epilogue.
#include <cuda_bf16.h>

#include "internal.h"
#include "learned.h"
#include "umma.cuh"

namespace isg {

constexpr int kGemmThreads = 128;
constexpr int kGemmKC = 64;
constexpr uint32_t kGemmWaitPolls = 1u << 22;

__device__ __forceinline__ float gelu_tanh(float x) {
    const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
    return 0.5f * x * (1.f + tanhf(u));
}

__global__ void __launch_bounds__(kGemmThreads) k_gemm_bf16(const GemmArgs g) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int N = g.N;
    const uint32_t a_bytes = 128u * kGemmKC * 2u;
    const uint32_t b_bytes = (uint32_t)N * kGemmKC * 2u;
    const uint32_t stage_bytes = a_bytes + b_bytes;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 2 * stage_bytes);
    uint32_t* slot = reinterpret_cast<uint32_t*>(smem + 2 * stage_bytes + 16);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * 128;
    const uint32_t ncols = g.tmem_cols;

    if (warp == 0) tmem_alloc(slot, ncols);
    if (tid == 0) { mbar_init(&bar[0], 1); mbar_init(&bar[1], 1); mbar_init_fence(); }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t taddr = *slot;
    const uint32_t idesc = umma_idesc_bf16(128, N);
    const int nk = (g.K + kGemmKC - 1) / kGemmKC;
    bool ok = true;
    for (int c = 0; c < nk && ok; ++c) {
        const int s = c & 1;
        if (c >= 2) ok = mbar_wait(&bar[s], (uint32_t)(((c - 2) >> 1) & 1), kGemmWaitPolls);
        if (!__syncthreads_and(ok)) { ok = false; break; }
        unsigned char* sA = smem + s * stage_bytes;
        unsigned char* sB = sA + a_bytes;
        const int kc0 = c * kGemmKC;
        const int kw = min(kGemmKC, g.K - kc0);   // multiple of 16
        const int q8 = kw >> 3;
        for (int i = tid; i < 128 * q8; i += kGemmThreads) {
            const int r = i / q8, q = i - r * q8;
            const int row = m0 + r, k = kc0 + 8 * q;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (g.conv_in) {
                // implicit convolution: the 8 values are channels ch..ch+7 of kernel offset o
                const int C = g.conv_C, Go = g.conv_Go, Gi = g.conv_Gi;
                const int o = k / C, ch = k - o * C;
                if (row < g.M && o < 27) {
                    const int Go3 = Go * Go * Go;
                    const int b = row / Go3, u = row - b * Go3;
                    const int x = u / (Go * Go) + o / 9 - g.conv_pad;
                    const int y = (u / Go) % Go + (o / 3) % 3 - g.conv_pad;
                    const int z = u % Go + o % 3 - g.conv_pad;
                    if (x >= 0 && x < Gi && y >= 0 && y < Gi && z >= 0 && z < Gi)
                        v = *reinterpret_cast<const uint4*>(g.conv_in + ((((int64_t)b * Gi + x) * Gi + y) * Gi + z) * C + ch);
                }
            } else {
                v = *reinterpret_cast<const uint4*>(g.A + (size_t)row * g.lda + k);
            }
            *reinterpret_cast<uint4*>(sA + umma_off(128, r, 8 * q)) = v;
        }
        for (int i = tid; i < N * q8; i += kGemmThreads) {
            const int r = i / q8, q = i - r * q8;
            const uint4 v = *reinterpret_cast<const uint4*>(g.B + (size_t)r * g.ldb + kc0 + 8 * q);
            *reinterpret_cast<uint4*>(sB + umma_off(N, r, 8 * q)) = v;
        }
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
            for (int j = 0; j < (kw >> 4); ++j) {
                const uint64_t ad = umma_smem_desc(a0 + (uint32_t)(2 * j) * (128u * 16u), 128u * 16u, 128u);
                const uint64_t bd = umma_smem_desc(b0 + (uint32_t)(2 * j) * ((uint32_t)N * 16u), (uint32_t)N * 16u, 128u);
                umma_bf16(taddr, ad, bd, idesc, (c > 0 || j > 0) ? 1u : 0u);
            }
            umma_commit(&bar[s]);
        }
    }
    if (ok) ok = mbar_wait(&bar[(nk - 1) & 1], (uint32_t)(((nk - 1) >> 1) & 1), kGemmWaitPolls);
    ok = __syncthreads_and(ok);
    tc_fence_after();
    if (!ok) {
        if (tid == 0) atomicOr(g.status, kStatTimeout);
    } else {
        const int row = m0 + warp * 32 + lane;
        for (int cb = 0; cb < N; cb += 32) {
            float v[32];
            tmem_ld32(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)cb, v);
            if (row < g.M) {
                const int nc = min(32, N - cb);
                for (int i = 0; i < nc; ++i) {
                    float x = v[i] + (g.bias ? g.bias[cb + i] : 0.f);
                    if (g.C) g.C[(size_t)row * g.ldc + cb + i] = g.accumulate ? g.C[(size_t)row * g.ldc + cb + i] + x : x;
                    if (g.O) g.O[(size_t)row * g.ldo + cb + i] = __float2bfloat16_rn(g.gelu ? gelu_tanh(x) : x);
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(taddr, ncols);
}

static int gemm_smem_bytes(int N) { return 2 * (128 * kGemmKC * 2 + N * kGemmKC * 2) + 64; }

int launch_gemm_bf16(GemmArgs g, cudaStream_t s) {
    if (g.N < 16 || g.N > 256 || g.N % 16) return fail(ISING_ERR_ARG, "GEMM N must be a multiple of 16 in 16..256");
    if (g.K < 16 || g.K % 16) return fail(ISING_ERR_ARG, "GEMM K must be a positive multiple of 16");
    if (g.M < 1) return ISING_OK;
    if (g.conv_in) {
        if (g.conv_C % 8 || g.K != 27 * g.conv_C || g.conv_Gi < 1 || g.conv_Go < 1)
            return fail(ISING_ERR_ARG, "implicit convolution needs C % 8 == 0 and K = 27 C");
        if (reinterpret_cast<uintptr_t>(g.conv_in) & 15) return fail(ISING_ERR_ARG, "GEMM operands must be 16-byte aligned");
    } else {
        if (g.lda % 8 || g.lda < g.K) return fail(ISING_ERR_ARG, "GEMM row pitch must be >= K and a multiple of 8");
        if (reinterpret_cast<uintptr_t>(g.A) & 15) return fail(ISING_ERR_ARG, "GEMM operands must be 16-byte aligned");
    }
    if (g.ldb % 8 || g.ldb < g.K) return fail(ISING_ERR_ARG, "GEMM row pitch must be >= K and a multiple of 8");
    if (reinterpret_cast<uintptr_t>(g.B) & 15) return fail(ISING_ERR_ARG, "GEMM operands must be 16-byte aligned");
    g.tmem_cols = g.N <= 32 ? 32 : g.N <= 64 ? 64 : g.N <= 128 ? 128 : 256;
    // resident blocks per SM x TMEM columns must fit the SM's 512 columns: a block whose
    // allocation cannot be met would stall until another block frees its columns
    int smem = gemm_smem_bytes(g.N);
    static bool attr_set = false;
    if (!attr_set) {
        ISG_CUDA(cudaFuncSetAttribute(k_gemm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        attr_set = true;
    }
    for (;;) {
        int occ = 0;
        ISG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_gemm_bf16, kGemmThreads, smem));
        if (occ * (int)g.tmem_cols <= 512 || smem >= 200 * 1024) break;
        smem += 8 * 1024;
    }
    const int grid = (g.M + 127) / 128;
    k_gemm_bf16<<<grid, kGemmThreads, smem, s>>>(g);
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}

static __device__ int g_gemm_status;

}  // namespace isg

using namespace isg;

extern "C" int ising_bf16_gemm(const void* a, int lda, const void* b, int ldb, int M, int N, int K, const float* bias,
                               float* c, int ldc, void* o_bf16, int ldo, int gelu, void* stream) {
    if (!a || !b || (!c && !o_bf16)) return fail(ISING_ERR_ARG, "NULL operand");
    int* st = nullptr;
    ISG_CUDA(cudaGetSymbolAddress((void**)&st, g_gemm_status));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ISG_CUDA(cudaMemsetAsync(st, 0, sizeof(int), s));
    GemmArgs g{};
    g.A = static_cast<const __nv_bfloat16*>(a); g.lda = lda;
    g.B = static_cast<const __nv_bfloat16*>(b); g.ldb = ldb;
    g.M = M; g.N = N; g.K = K; g.bias = bias; g.C = c; g.ldc = ldc; g.accumulate = 0;
    g.O = static_cast<__nv_bfloat16*>(o_bf16); g.ldo = ldo; g.gelu = gelu; g.status = st;
    int r = launch_gemm_bf16(g, s);
    if (r != ISING_OK) return r;
    int h = 0;
    ISG_CUDA(cudaMemcpyAsync(&h, st, sizeof(int), cudaMemcpyDeviceToHost, s));
    ISG_CUDA(cudaStreamSynchronize(s));
    if (h & kStatTimeout) return fail(ISING_ERR_TIMEOUT, "tensor-core GEMM: an mbarrier wait gave up");
    return ISING_OK;
}
