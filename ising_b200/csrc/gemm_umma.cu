// gemm_umma.cu -- C = A * B^T on the sm_100a tensor cores (tcgen05.mma kind::f16, BF16 in,
// FP32 accumulation in TMEM), the matrix engine of the learned patch proposal: every
// convolution of its forward and backward passes is an im2col matrix times a weight matrix.
//
// A is M x K, B is N x K, both BF16 with K contiguous (row pitches lda, ldb, multiples of
// 8 elements), K a multiple of 16, N a multiple of 16 up to 256; A holds ceil(M/128)*128
// readable rows.  For a 3^3 convolution over an 8- or 32-channel grid A is not stored: the
// loader gathers its 16-byte pieces from the channel-last input grid (implicit GEMM), zero
// outside the grid.  Blocks have 256 threads: two per tile row (each loads half of the row's
// pieces of a K chunk, prefetched one chunk ahead in registers; the row is decomposed once
// before the K loop), and in the epilogue the two warps of a TMEM lane quadrant split each
// 32-column block.  One block computes a 128-row tile for all N columns:
// chunks of 64 values of K are staged by all threads into a two-stage ring in the canonical
// no-swizzle layout (umma.cuh), thread 0 issues the MMAs and commits them to the stage's
// mbarrier, and the block refills a stage once that mbarrier reports its MMAs done.  The
// epilogue reads each thread's TMEM lane (one output row), adds the bias, applies GELU when
// asked, and stores FP32 and/or BF16 rows.  Every mbarrier wait is bounded; a wait that
// gives up sets kStatTimeout and skips the epilogue.
#include <cuda_bf16.h>

#include <atomic>

#include "internal.h"
#include "learned.h"
#include "umma.cuh"

namespace isg {

constexpr int kGemmThreads = 256;   // two threads per row of the 128-row tile
constexpr int kGemmKC = 64;
constexpr uint32_t kGemmWaitPolls = 1u << 22;

__device__ __forceinline__ float gelu_tanh(float x) {
    const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
    return 0.5f * x * (1.f + tanhf(u));
}

__global__ void __launch_bounds__(kGemmThreads, 4) k_gemm_bf16(const GemmArgs g) {
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
    // implicit convolution: this thread's row is fixed for the whole K loop
    const __nv_bfloat16* cbase = nullptr;
    int cx = 0, cy = 0, cz = 0;
    bool crow_ok = false;
    if (g.conv_in) {
        const int row = m0 + (tid & 127), Go = g.conv_Go, Gi = g.conv_Gi;
        const int Go3 = Go * Go * Go;
        crow_ok = row < g.M;
        const int b = crow_ok ? row / Go3 : 0, u = crow_ok ? row - b * Go3 : 0;
        cx = u / (Go * Go) - g.conv_pad;
        cy = (u / Go) % Go - g.conv_pad;
        cz = u % Go - g.conv_pad;
        cbase = g.conv_in + (int64_t)b * Gi * Gi * Gi * g.conv_C;
    }
    const bool C32 = g.conv_C == 32;
    // Register-staged pipeline: the loads of chunk c+1 are issued right after chunk c is
    // stored to shared memory, so they are in flight while chunk c's MMAs are issued and
    // the next stage is awaited.  A: this thread's row, 8 values per piece, q8 <= 8 pieces;
    // B: N x q8 pieces spread over the block (<= 16 per thread).
    uint4 va[4], vb[8];
    const int arow = tid & 127, ahalf = tid >> 7;   // this thread's A row and half of the pieces
    auto load_chunk = [&](int c) {
        const int kc0 = c * kGemmKC;
        const int q8 = min(kGemmKC, g.K - kc0) >> 3;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int j = ahalf + 2 * i;
            va[i] = make_uint4(0u, 0u, 0u, 0u);
            if (j < q8) {
                const int k = kc0 + 8 * j;
                if (g.conv_in) {
                    // implicit convolution: channels ch..ch+7 of kernel offset o of this row's voxel
                    const int o = C32 ? (k >> 5) : (k >> 3), ch = C32 ? (k & 31) : 0;
                    if (crow_ok && o < 27) {
                        const int x = cx + o / 9, y = cy + (o / 3) % 3, z = cz + o % 3;
                        const int Gi = g.conv_Gi;
                        if ((unsigned)x < (unsigned)Gi && (unsigned)y < (unsigned)Gi && (unsigned)z < (unsigned)Gi)
                            va[i] = *reinterpret_cast<const uint4*>(cbase + (((int64_t)x * Gi + y) * Gi + z) * g.conv_C + ch);
                    }
                } else {
                    va[i] = *reinterpret_cast<const uint4*>(g.A + (size_t)(m0 + arow) * g.lda + k);
                }
            }
        }
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) {
            const int i = tid + jj * kGemmThreads;
            if (i < N * q8) {
                const int r = i / q8, q = i - r * q8;
                vb[jj] = *reinterpret_cast<const uint4*>(g.B + (size_t)r * g.ldb + kc0 + 8 * q);
            }
        }
    };
    auto store_chunk = [&](int c, unsigned char* sA, unsigned char* sB) {
        const int q8 = min(kGemmKC, g.K - c * kGemmKC) >> 3;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int j = ahalf + 2 * i;
            if (j < q8) *reinterpret_cast<uint4*>(sA + umma_off(128, arow, 8 * j)) = va[i];
        }
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) {
            const int i = tid + jj * kGemmThreads;
            if (i < N * q8) {
                const int r = i / q8, q = i - r * q8;
                *reinterpret_cast<uint4*>(sB + umma_off(N, r, 8 * q)) = vb[jj];
            }
        }
    };
    bool ok = true;
    load_chunk(0);
    for (int c = 0; c < nk && ok; ++c) {
        const int s = c & 1;
        if (c >= 2) ok = mbar_wait(&bar[s], (uint32_t)(((c - 2) >> 1) & 1), kGemmWaitPolls);
        if (!__syncthreads_and(ok)) { ok = false; break; }
        unsigned char* sA = smem + s * stage_bytes;
        unsigned char* sB = sA + a_bytes;
        store_chunk(c, sA, sB);
        if (c + 1 < nk) load_chunk(c + 1);
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const int kw = min(kGemmKC, g.K - c * kGemmKC);
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
        // epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 (one output row per thread) and the
        // 16-column half w / 4 of every 32-column block; 16-byte stores (ldc % 4 == 0, ldo % 8 == 0)
        const int quad = warp & 3, hcol = (warp >> 2) * 16;
        const int row = m0 + quad * 32 + lane;
        for (int cb = hcol; cb < N; cb += 32) {
            float v[16];
            tmem_ld16(taddr + ((uint32_t)(quad * 32) << 16) + (uint32_t)cb, v);
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
                if (g.O) {
                    uint4* op = reinterpret_cast<uint4*>(g.O + (size_t)row * g.ldo + cb);
#pragma unroll
                    for (int q = 0; q < 2; ++q) {
                        uint32_t w[4];
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const float a = g.gelu ? gelu_tanh(v[8 * q + 2 * e]) : v[8 * q + 2 * e];
                            const float b = g.gelu ? gelu_tanh(v[8 * q + 2 * e + 1]) : v[8 * q + 2 * e + 1];
                            const __nv_bfloat162 h2 = __floats2bfloat162_rn(a, b);
                            w[e] = *reinterpret_cast<const uint32_t*>(&h2);
                        }
                        op[q] = make_uint4(w[0], w[1], w[2], w[3]);
                    }
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
        if ((g.conv_C != 8 && g.conv_C != 32) || g.K < 27 * g.conv_C || g.K > 27 * g.conv_C + 15 || g.conv_Gi < 1 ||
            g.conv_Go < 1)
            return fail(ISING_ERR_ARG, "implicit convolution needs C = 8 or 32 and K = 27 C rounded up to 16");
        if (reinterpret_cast<uintptr_t>(g.conv_in) & 15) return fail(ISING_ERR_ARG, "GEMM operands must be 16-byte aligned");
    } else {
        if (g.lda % 8 || g.lda < g.K) return fail(ISING_ERR_ARG, "GEMM row pitch must be >= K and a multiple of 8");
        if (reinterpret_cast<uintptr_t>(g.A) & 15) return fail(ISING_ERR_ARG, "GEMM operands must be 16-byte aligned");
    }
    if (g.ldb % 8 || g.ldb < g.K) return fail(ISING_ERR_ARG, "GEMM row pitch must be >= K and a multiple of 8");
    if (reinterpret_cast<uintptr_t>(g.B) & 15) return fail(ISING_ERR_ARG, "GEMM operands must be 16-byte aligned");
    if (g.C && (g.ldc % 4 || g.ldc < g.N || (reinterpret_cast<uintptr_t>(g.C) & 15)))
        return fail(ISING_ERR_ARG, "GEMM FP32 output needs a 16-byte aligned base and ldc % 4 == 0");
    if (g.O && (g.ldo % 8 || g.ldo < g.N || (reinterpret_cast<uintptr_t>(g.O) & 15)))
        return fail(ISING_ERR_ARG, "GEMM BF16 output needs a 16-byte aligned base and ldo % 8 == 0");
    if (g.loader == 2 || (g.loader == 0 && conv_tma_applies(g))) return launch_conv_tma(g, s);
    if (g.head_out) return fail(ISING_ERR_ARG, "the fused head needs the TMA convolution path");
    g.tmem_cols = g.N <= 32 ? 32 : g.N <= 64 ? 64 : g.N <= 128 ? 128 : 256;
    // resident blocks per SM x TMEM columns must fit the SM's 512 columns: a block whose
    // allocation cannot be met would stall until another block frees its columns
    int smem = gemm_smem_bytes(g.N);
    // the shared-memory limit is a per-device attribute of the kernel: raise it once per device
    static std::atomic<unsigned long long> attr_set{0};
    {
        int dev = 0;
        ISG_CUDA(cudaGetDevice(&dev));
        const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
        if (!bit || !(attr_set.load() & bit)) {
            ISG_CUDA(cudaFuncSetAttribute(k_gemm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
            attr_set.fetch_or(bit);
        }
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

extern "C" int ising_conv3_bf16(const void* in, int C, int Gi, int Go, int pad, int nwin, const void* w, int ldb, int N,
                                const float* bias, float* c, int ldc, void* o_bf16, int ldo, int gelu, int loader,
                                void* stream) {
    if (!in || !w || (!c && !o_bf16)) return fail(ISING_ERR_ARG, "NULL operand");
    if (nwin < 1 || loader < 0 || loader > 2) return fail(ISING_ERR_ARG, "bad window count or loader");
    int* st = nullptr;
    ISG_CUDA(cudaGetSymbolAddress((void**)&st, g_gemm_status));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ISG_CUDA(cudaMemsetAsync(st, 0, sizeof(int), s));
    GemmArgs g{};
    g.B = static_cast<const __nv_bfloat16*>(w); g.ldb = ldb;
    g.M = nwin * Go * Go * Go; g.N = N; g.K = (27 * C + 15) / 16 * 16; g.bias = bias; g.C = c; g.ldc = ldc;
    g.O = static_cast<__nv_bfloat16*>(o_bf16); g.ldo = ldo; g.gelu = gelu; g.status = st;
    g.conv_in = static_cast<const __nv_bfloat16*>(in); g.conv_C = C; g.conv_Gi = Gi; g.conv_Go = Go; g.conv_pad = pad;
    g.loader = loader;
    int r = launch_gemm_bf16(g, s);
    if (r != ISING_OK) return r;
    int h = 0;
    ISG_CUDA(cudaMemcpyAsync(&h, st, sizeof(int), cudaMemcpyDeviceToHost, s));
    ISG_CUDA(cudaStreamSynchronize(s));
    if (h & kStatTimeout) return fail(ISING_ERR_TIMEOUT, "tensor-core convolution: an mbarrier wait gave up");
    return ISING_OK;
}

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
