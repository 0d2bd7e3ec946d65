// learned.h -- device-side interfaces of the learned patch proposal (tensor-core GEMM and
// the network kernels).
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

#include "internal.h"

namespace isg {

// C/O[M x N] = epilogue(A[M x K] * B[N x K]^T + bias)
struct GemmArgs {
    const __nv_bfloat16* A;
    int lda;
    const __nv_bfloat16* B;
    int ldb;
    int M, N, K;
    const float* bias;      // [N] or null
    float* C;               // FP32 rows (acc + bias), or null
    int ldc;
    int accumulate;         // C += instead of C =
    __nv_bfloat16* O;       // BF16 rows: gelu(acc + bias) when gelu, else acc + bias; or null
    int ldo;
    int gelu;
    int* status;
    uint32_t tmem_cols;     // set by the launcher
};
int launch_gemm_bf16(GemmArgs g, cudaStream_t s);

}  // namespace isg
