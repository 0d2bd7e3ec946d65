// learned.h -- device-side interfaces of the learned patch proposal (tensor-core GEMM and
// the network kernels).
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

#include "internal.h"

struct ising_net;

namespace isg {

// range of log sigma in the proposal and in the training loss
constexpr float kLogSigMin = -6.f, kLogSigMax = 1.5f;

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
    // implicit convolution: when conv_in is set, A is not read; A(row, k) = conv_in[b][u + o -
    // conv_pad][c] for row = b*Go^3 + u, k = o*C + c (C = 8 or 32), zero outside the grid, for
    // o >= 27 or for row >= M
    const __nv_bfloat16* conv_in;
    int conv_C, conv_Gi, conv_Go, conv_pad;
    // operand path: 0 = TMA copies where the shape allows (conv_tma.cu), else registers;
    // 1 = register-staged loader; 2 = TMA copies (an error where the shape does not allow)
    int loader;
    // optional 1^3 head fused into the TMA path's epilogue (32 -> 4 channels onto 4^3 grids):
    // head_out[row][o] = head_b[o] + sum_c bf16(gelu(acc + bias))[row][c] head_w[o][c], the
    // channels taken in order; the register path refuses it
    const float* head_w;
    const float* head_b;
    float* head_out;
    uint32_t tmem_cols;     // set by the launcher
};
int launch_gemm_bf16(GemmArgs g, cudaStream_t s);
// 3^3 convolution over 32 channels onto a 4^3 output grid (pad 0 from 6^3, pad 1 from 4^3)
// with TMA-fed operands (conv_tma.cu)
bool conv_tma_applies(const GemmArgs& g);
int launch_conv_tma(const GemmArgs& g, cudaStream_t s);

// the network's input-row buffer ([max_batch*512][8] BF16) and a forward on stream s of the
// nb windows already written there; *out = [nb*64][4]
__nv_bfloat16* net_rows(ising_net* n);
int net_forward_prepared(ising_net* n, int nb, cudaStream_t s, const float** out);
int net_max_batch(const ising_net* n);
int net_device(const ising_net* n);
// reads and clears the network status word after the work queued on s (synchronises s)
int net_status_on(ising_net* n, cudaStream_t s);

// One class of the 2x2x2 colouring of 4^3 blocks (shifted by (offx, offy, offz)) on the
// replicas that hold temperature slots 0..n_slots-1: window w belongs to slot w / per_slot.
struct PatchStep {
    float* spins;
    int64_t natoms;
    int nx, ny, nz;
    Layout layout;
    int colour, offx, offy, offz;
    int per_slot;
    const int* t2r;            // slot -> replica
    const double* beta_rep;
    const float* step_scale;   // per slot: the tangent move is scale * (drift P_s(mu) + sigma eps); null = 1
    float drift;               // weight of the network's mean rotation (1 = the mean as predicted)
    HamDev ham;
    uint64_t seed;
    uint32_t ensemble;
    uint32_t round;
    int* status;
};
// windows w0 .. w0+nb-1 as FP32 [window][3][512] in win and, when x0 is given, as the
// network's BF16 input rows (net_rows) for net_forward_prepared
int launch_patch_gather(const PatchStep& P, int64_t w0, int nb, const float* prop, float* win, cudaStream_t s,
                        __nv_bfloat16* x0 = nullptr);
int launch_patch_propose(const PatchStep& P, int64_t w0, int nb, const float* win, const float* out, float* prop,
                         double* lqf, int* rej, cudaStream_t s);
int launch_patch_accept(const PatchStep& P, int64_t w0, int nb, const float* win, const float* winp, const float* outp,
                        const float* prop, const double* lqf, const int* rej, double* dE, double* dM4, int* acc,
                        cudaStream_t s);
int launch_patch_fold(const PatchStep& P, int n_slots, int64_t n_windows, const double* dE, const double* dM,
                      const int* accepted, Acc4* acc, unsigned long long* stats, double* jump, cudaStream_t s);
int launch_patch_equilibrate(const PatchStep& P, int64_t w0, int nb, const float* win, int n_local, int move, float r,
                             float* tgt, cudaStream_t s);

}  // namespace isg
