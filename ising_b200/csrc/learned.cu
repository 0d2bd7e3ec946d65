// learned.cu -- the proposal network of the learned patch move: forward, backward and Adam
// on the tensor cores (gemm_umma.cu), everything else on CUDA cores.
//
// Network (per 8^3 window of 3-component spins): conv 3->32 (3^3, valid, 8^3 -> 6^3), conv
// 32->32 (valid, 6^3 -> 4^3), conv 32->32 (3^3, zero padding, 4^3 -> 4^3), GELU (tanh form)
// after each, then a 1^3 head 32 -> 4 giving mu (3) and log sigma per patch site.
// Activations are channel-last BF16 rows (one row per window voxel); each convolution is
//     out[rows x 32] = im2col(in)[rows x 27*Cin] * Wf[32 x 27*Cin]^T + b      (tensor cores)
// where im2col(in) is gathered inside the GEMM's loader (implicit GEMM; the 3 input channels
// are padded to 8, one 16-byte piece per voxel) and only the weight gradients use
// materialised (transposed) im2col matrices.
// with column k = o * Cin + c, o = (dx*3 + dy)*3 + dz.  Backward: the data gradient of a
// convolution is a convolution of the output gradient with the flipped, transposed kernel
// (same im2col, weights WfT[ci][o'*32 + co] = W[co][ci][26 - o']); the weight gradient is
// im2col(in)^T [27*Cin x rows] times dPre^T [32 x rows]^T.  Parameters are FP32 master
// copies (PyTorch conv3d order W[co][ci][dx][dy][dz]) updated by Adam; the BF16 operand
// matrices are repacked after every update.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <vector>

#include "learned.h"

#define ISG_TRY_N(expr)                   \
    do {                                  \
        int st_ = (expr);                 \
        if (st_ != ISING_OK) return st_;  \
    } while (0)
#ifndef ISG_TRY
#define ISG_TRY(expr) ISG_TRY_N(expr)
#endif

namespace isg {

constexpr int kCh = 32;
constexpr int kC0 = 8;            // input channels padded to 8 (one 16-byte piece per voxel)
constexpr int kK1 = 224;          // 27 * 8 = 216 padded to a multiple of 16
constexpr int kK2 = 27 * kCh;     // 864
constexpr int kK2Pad = 896;       // rows of the transposed im2col for weight gradients
constexpr int kOffW1 = 0, kOffB1 = 2592, kOffW2 = 2624, kOffB2 = 30272, kOffW3 = 30304, kOffB3 = 57952,
              kOffWh = 57984, kOffBh = 58112, kNParams = 58116;

static inline size_t pad32(size_t n) { return (n + 31) / 32 * 32; }

__device__ __forceinline__ float gelu_f(float x) {
    const float u = 0.7978845608028654f * (x + 0.044715f * x * x * x);
    return 0.5f * x * (1.f + tanhf(u));
}
__device__ __forceinline__ float gelu_d(float x) {
    const float k = 0.7978845608028654f;
    const float t = tanhf(k * (x + 0.044715f * x * x * x));
    return 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * k * (1.f + 3.f * 0.044715f * x * x);
}

// ---------------------------------------------------------------- layout kernels
// windows [B][3][8][8][8] FP32 -> X0 rows [B*512][8] BF16 (channels 3..7 zero)
__global__ void k_windows_to_rows(const float* __restrict__ w, int nb, __nv_bfloat16* __restrict__ x0) {
    const int64_t n = (int64_t)nb * 512;
    for (int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; row < n; row += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = row / 512;
        const int v = (int)(row - b * 512);
        __nv_bfloat162 h[4];
        h[0] = __floats2bfloat162_rn(w[(b * 3 + 0) * 512 + v], w[(b * 3 + 1) * 512 + v]);
        h[1] = __floats2bfloat162_rn(w[(b * 3 + 2) * 512 + v], 0.f);
        h[2] = __floats2bfloat162_rn(0.f, 0.f);
        h[3] = h[2];
        *reinterpret_cast<uint4*>(x0 + row * kC0) = *reinterpret_cast<const uint4*>(h);
    }
}

// im2col of channel-last rows in[b][Gi^3][C]: element (row, k) = in[b][u + o - pad][c] for
// row = b*Go^3 + u, k = o*C + c < 27C, zero outside the input grid and for k >= 27C.
// Plain: out[row * Kp + k] for rows < n_rows.  Transposed: out[k * ldt + row] for k < Kt and
// row < ldt (zero beyond n_rows or 27C).
__global__ void k_im2col(const __nv_bfloat16* __restrict__ in, int C, int Gi, int Go, int pad, int64_t n_rows,
                         __nv_bfloat16* __restrict__ out, int Kp, int transpose, int64_t ldt, int Kt) {
    const int Go3 = Go * Go * Go;
    const int64_t total = transpose ? (int64_t)Kt * ldt : n_rows * Kp;
    const __nv_bfloat16 zero = __float2bfloat16_rn(0.f);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t row;
        int k;
        if (transpose) { k = (int)(i / ldt); row = i - (int64_t)k * ldt; }
        else { row = i / Kp; k = (int)(i - row * Kp); }
        __nv_bfloat16 v = zero;
        if (row < n_rows && k < 27 * C) {
            const int o = k / C, c = k - o * C;
            const int dx = o / 9, dy = (o / 3) % 3, dz = o % 3;
            const int64_t b = row / Go3;
            const int u = (int)(row - b * Go3);
            const int x = u / (Go * Go) + dx - pad, y = (u / Go) % Go + dy - pad, z = u % Go + dz - pad;
            if (x >= 0 && x < Gi && y >= 0 && y < Gi && z >= 0 && z < Gi)
                v = in[((b * Gi + x) * Gi + y) * (int64_t)Gi * C + (int64_t)z * C + c];
        }
        out[i] = v;
    }
}

// BF16 operand matrices from the FP32 parameters
__global__ void k_pack(const float* __restrict__ P, __nv_bfloat16* Wf1, __nv_bfloat16* Wf2, __nv_bfloat16* Wf3,
                       __nv_bfloat16* W2fT, __nv_bfloat16* W3fT) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kCh * kK1) {
        const int co = i / kK1, k = i % kK1;
        float v = 0.f;
        const int o = k / kC0, c = k % kC0;
        if (o < 27 && c < 3) v = P[kOffW1 + (co * 3 + c) * 27 + o];
        Wf1[i] = __float2bfloat16_rn(v);
    }
    if (i < kCh * kK2) {
        const int r = i / kK2, k = i % kK2, o = k / kCh, c = k % kCh;
        // forward: row co = r, column (o, ci = c); backward-data: row ci = r, column (o', co = c)
        Wf2[i] = __float2bfloat16_rn(P[kOffW2 + (r * kCh + c) * 27 + o]);
        Wf3[i] = __float2bfloat16_rn(P[kOffW3 + (r * kCh + c) * 27 + o]);
        W2fT[i] = __float2bfloat16_rn(P[kOffW2 + (c * kCh + r) * 27 + (26 - o)]);
        W3fT[i] = __float2bfloat16_rn(P[kOffW3 + (c * kCh + r) * 27 + (26 - o)]);
    }
}

// head: out[row][o] = sum_c H3[row][c] Wh[o][c] + bh[o]
__global__ void k_head_fwd(const __nv_bfloat16* __restrict__ h3, int64_t rows, const float* __restrict__ P,
                           float* __restrict__ out) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (r >= rows) return;
    float a[4] = {P[kOffBh], P[kOffBh + 1], P[kOffBh + 2], P[kOffBh + 3]};
    for (int c = 0; c < kCh; ++c) {
        const float h = __bfloat162float(h3[r * kCh + c]);
        for (int o = 0; o < 4; ++o) a[o] = fmaf(h, P[kOffWh + o * kCh + c], a[o]);
    }
    for (int o = 0; o < 4; ++o) out[r * 4 + o] = a[o];
}

// ---------------------------------------------------------------- tangent geometry
struct F3 { float x, y, z; };
__device__ __forceinline__ F3 f3(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ F3 cross3(F3 a, F3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
__device__ __forceinline__ F3 axpy3(float a, F3 x, F3 y) { return {a * x.x + y.x, a * x.y + y.y, a * x.z + y.z}; }
__device__ __forceinline__ F3 scale3(float a, F3 x) { return {a * x.x, a * x.y, a * x.z}; }

// tangent frame at s: helper axis z (x when |s_z| >= 0.9), e1 = normalize(a x s), e2 = s x e1
__device__ __forceinline__ void tframe(F3 s, F3& e1, F3& e2) {
    const F3 a = fabsf(s.z) >= 0.9f ? f3(1.f, 0.f, 0.f) : f3(0.f, 0.f, 1.f);
    e1 = cross3(a, s);
    e1 = scale3(rsqrtf(dot3(e1, e1)), e1);
    e2 = cross3(s, e1);
}
// log_s(t) in the frame of s; returns the angle
__device__ __forceinline__ float tlog(F3 s, F3 t, float& w1, float& w2) {
    const float c = fminf(1.f, fmaxf(-1.f, dot3(s, t)));
    const F3 v = axpy3(-c, s, t);
    const float nv = sqrtf(dot3(v, v));
    const float th = atan2f(nv, c);   // small angles keep their bits (acos of c near 1 would not)
    F3 e1, e2;
    tframe(s, e1, e2);
    const float sc = nv > 1e-12f ? th / nv : 0.f;
    w1 = sc * dot3(v, e1);
    w2 = sc * dot3(v, e2);
    return th;
}

// per-site Gaussian NLL of the target rotation and its gradient wrt (mu, log sigma);
// windows [B][3][8][8][8] FP32 give the current patch spins, targets [B][64][3]
__global__ void k_nll(const float* __restrict__ win, const float* __restrict__ tgt, const float* __restrict__ out,
                      int64_t rows, float inv_n, float* __restrict__ dout, double* __restrict__ loss_acc) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double l = 0.0;
    if (r < rows) {
        const int64_t b = r / 64;
        const int i = (int)(r - b * 64);
        const int x = i / 16 + 2, y = (i / 4) % 4 + 2, z = i % 4 + 2;
        const int v = (x * 8 + y) * 8 + z;
        const F3 s = f3(win[(b * 3 + 0) * 512 + v], win[(b * 3 + 1) * 512 + v], win[(b * 3 + 2) * 512 + v]);
        const F3 t = f3(tgt[r * 3], tgt[r * 3 + 1], tgt[r * 3 + 2]);
        float w1, w2;
        tlog(s, t, w1, w2);
        F3 e1, e2;
        tframe(s, e1, e2);
        const F3 mu = f3(out[r * 4], out[r * 4 + 1], out[r * 4 + 2]);
        // log sigma clamped to the range the proposal uses (a target that did not move would
        // otherwise drive log sigma to -infinity and the loss to NaN); no gradient outside it
        const float lraw = out[r * 4 + 3];
        const float ls = fminf(kLogSigMax, fmaxf(kLogSigMin, lraw));
        const float r1 = w1 - dot3(mu, e1), r2 = w2 - dot3(mu, e2);
        const float is2 = expf(-2.f * ls);
        const float q = r1 * r1 + r2 * r2;
        l = 0.5 * (double)q * is2 + 2.0 * ls;
        // d/dmu = -(r1 e1 + r2 e2) / sigma^2 ; d/dlog sigma = -q / sigma^2 + 2
        const F3 g = scale3(-is2 * inv_n, axpy3(r1, e1, scale3(r2, e2)));
        dout[r * 4] = g.x; dout[r * 4 + 1] = g.y; dout[r * 4 + 2] = g.z;
        dout[r * 4 + 3] = (lraw > kLogSigMin && lraw < kLogSigMax) ? (-q * is2 + 2.f) * inv_n : 0.f;
    }
    l = warp_sum(l);
    if ((threadIdx.x & 31) == 0 && l != 0.0) atomicAdd(loss_acc, l);
}

// head backward: dH3 = dOut Wh (FP32 rows), dWh += dOut^T H3, dbh += sum dOut
__global__ void k_head_bwd(const float* __restrict__ dout, const __nv_bfloat16* __restrict__ h3, int64_t rows,
                           const float* __restrict__ P, float* __restrict__ dh, float* __restrict__ G) {
    const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    float gd[4] = {0, 0, 0, 0};
    float d[4] = {0, 0, 0, 0};
    if (r < rows) for (int o = 0; o < 4; ++o) d[o] = dout[r * 4 + o];
    for (int c = 0; c < kCh; ++c) {
        const float h = r < rows ? __bfloat162float(h3[r * kCh + c]) : 0.f;
        if (r < rows) dh[r * kCh + c] = d[0] * P[kOffWh + c] + d[1] * P[kOffWh + kCh + c] +
                                        d[2] * P[kOffWh + 2 * kCh + c] + d[3] * P[kOffWh + 3 * kCh + c];
        for (int o = 0; o < 4; ++o) {
            const float v = warp_sum(d[o] * h);
            if (lane == 0) atomicAdd(&G[kOffWh + o * kCh + c], v);
        }
    }
    for (int o = 0; o < 4; ++o) gd[o] = warp_sum(d[o]);
    if (lane == 0) for (int o = 0; o < 4; ++o) atomicAdd(&G[kOffBh + o], gd[o]);
}

// dPre = dH * gelu'(pre): BF16 rows, BF16 transposed [32][ldt] (zero padded), bias gradient
__global__ void k_gelu_bwd(const float* __restrict__ dh, const float* __restrict__ pre, int64_t rows, int64_t ldt,
                           __nv_bfloat16* __restrict__ dp, __nv_bfloat16* __restrict__ dpt, float* __restrict__ gb) {
    // over 32 x ldt elements, channel-major; ldt % 32 == 0 and the stride is whole warps, so
    // every warp covers 32 rows of one channel and all its lanes take the same trip count
    const int64_t total = (int64_t)kCh * ldt;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i - (threadIdx.x & 31) < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(i / ldt);
        const int64_t r = i - (int64_t)c * ldt;
        float v = 0.f;
        if (r < rows) {
            v = dh[r * kCh + c] * gelu_d(pre[r * kCh + c]);
            dp[r * kCh + c] = __float2bfloat16_rn(v);
        }
        dpt[(int64_t)c * ldt + r] = __float2bfloat16_rn(v);
        const float s = warp_sum(v);
        if ((threadIdx.x & 31) == 0 && s != 0.f) atomicAdd(&gb[c], s);
    }
}

// weight gradient rows C[k][co] (k = o*stride + ci, ci < Cin) -> G[W][co][ci][o]
__global__ void k_scatter_wgrad(const float* __restrict__ Cm, int Cin, int stride, int off, float* __restrict__ G) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 27 * Cin * kCh) return;
    const int co = i % kCh, j = i / kCh, o = j / Cin, ci = j % Cin;
    G[off + (co * Cin + ci) * 27 + o] += Cm[(o * stride + ci) * kCh + co];
}

__global__ void k_adam(float* __restrict__ P, const float* __restrict__ G, float* __restrict__ m, float* __restrict__ v,
                       int n, float lr, float b1t, float b2t) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = G[i];
    const float mi = 0.9f * m[i] + 0.1f * g, vi = 0.999f * v[i] + 0.001f * g * g;
    m[i] = mi;
    v[i] = vi;
    P[i] -= lr * (mi / (1.f - b1t)) / (sqrtf(vi / (1.f - b2t)) + 1e-8f);
}

static int grid_for(int64_t n, int t = 256) { return (int)std::min<int64_t>((n + t - 1) / t, 148 * 32); }

}  // namespace isg

using namespace isg;

struct ising_net {
    int device = 0;
    cudaStream_t stream = nullptr;
    int max_batch = 0;
    float *P = nullptr, *G = nullptr, *M = nullptr, *V = nullptr;
    int adam_t = 0;
    __nv_bfloat16 *Wf1 = nullptr, *Wf2 = nullptr, *Wf3 = nullptr, *W2fT = nullptr, *W3fT = nullptr;
    __nv_bfloat16 *X0 = nullptr, *H1 = nullptr, *H2 = nullptr, *H3 = nullptr;
    float *pre1 = nullptr, *pre2 = nullptr, *pre3 = nullptr, *out = nullptr;
    float *dout = nullptr, *dh = nullptr, *Cw = nullptr;
    __nv_bfloat16 *dp = nullptr, *dpt = nullptr, *AT = nullptr;
    double* loss = nullptr;
    int* status = nullptr;
};

namespace {

struct NetGuard {
    int prev = -1;
    explicit NetGuard(int dev) { cudaGetDevice(&prev); if (prev != dev) cudaSetDevice(dev); }
    ~NetGuard() { int cur = -1; cudaGetDevice(&cur); if (prev >= 0 && cur != prev) cudaSetDevice(prev); }
};

template <typename T>
int nalloc(T** p, size_t n) {
    *p = nullptr;
    if (cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        return fail(ISING_ERR_ALLOC, "cudaMalloc failed for the proposal network");
    }
    return ISING_OK;
}

void net_free(ising_net* n) {
    void* ptrs[] = {n->P, n->G, n->M, n->V, n->Wf1, n->Wf2, n->Wf3, n->W2fT, n->W3fT, n->X0, n->H1,
                    n->H2, n->H3, n->pre1, n->pre2, n->pre3, n->out, n->dout, n->dh, n->Cw, n->dp, n->dpt,
                    n->AT, n->loss, n->status};
    for (void* p : ptrs) cudaFree(p);
    if (n->stream) cudaStreamDestroy(n->stream);
}

int net_check(ising_net* n) {
    int h = 0;
    if (cudaMemcpyAsync(&h, n->status, sizeof(int), cudaMemcpyDeviceToHost, n->stream) != cudaSuccess ||
        cudaStreamSynchronize(n->stream) != cudaSuccess)
        return cuda_fail(cudaGetLastError(), "proposal network");
    if (h) {
        cudaMemsetAsync(n->status, 0, sizeof(int), n->stream);
        if (h & kStatTimeout) return fail(ISING_ERR_TIMEOUT, "tensor-core GEMM: an mbarrier wait gave up");
        return fail(ISING_ERR_NAN, "proposal network produced a non-finite value");
    }
    return ISING_OK;
}

GemmArgs gemm(const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, int M, int N, int K, int* st) {
    GemmArgs g{};
    g.A = A; g.lda = lda; g.B = B; g.ldb = ldb; g.M = M; g.N = N; g.K = K; g.status = st;
    return g;
}

// a 3^3 convolution over C-channel (8 or 32) channel-last grids as an implicit GEMM: rows
// over the Go^3 output grid of every window, A gathered by the GEMM's loader; K = 27 C
// rounded up to a multiple of 16 (the extra columns are zero)
GemmArgs conv_gemm(const __nv_bfloat16* in, int C, int Gi, int Go, int pad, const __nv_bfloat16* W, int K, int rows,
                   int* st) {
    GemmArgs g{};
    g.B = W; g.ldb = K; g.M = rows; g.N = kCh; g.K = K; g.status = st;
    g.conv_in = in; g.conv_C = C; g.conv_Gi = Gi; g.conv_Go = Go; g.conv_pad = pad;
    return g;
}

// forward of nb windows already in X0 into out; keep_pre also stores the FP32 pre-activations
// that the backward pass needs
int net_forward_rows(ising_net* n, int nb, bool keep_pre) {
    cudaStream_t s = n->stream;
    const int64_t R1 = (int64_t)nb * 216, R2 = (int64_t)nb * 64;
    GemmArgs g = conv_gemm(n->X0, kC0, 8, 6, 0, n->Wf1, kK1, (int)R1, n->status);
    g.bias = n->P + kOffB1; g.C = keep_pre ? n->pre1 : nullptr; g.ldc = kCh; g.O = n->H1; g.ldo = kCh; g.gelu = 1;
    ISG_TRY_N(launch_gemm_bf16(g, s));
    g = conv_gemm(n->H1, kCh, 6, 4, 0, n->Wf2, kK2, (int)R2, n->status);
    g.bias = n->P + kOffB2; g.C = keep_pre ? n->pre2 : nullptr; g.ldc = kCh; g.O = n->H2; g.ldo = kCh; g.gelu = 1;
    ISG_TRY_N(launch_gemm_bf16(g, s));
    g = conv_gemm(n->H2, kCh, 4, 4, 1, n->Wf3, kK2, (int)R2, n->status);
    g.bias = n->P + kOffB3; g.C = keep_pre ? n->pre3 : nullptr; g.ldc = kCh; g.O = n->H3; g.ldo = kCh; g.gelu = 1;
    // the TMA path computes the head in its epilogue; H3 is then written only for training
    const bool fused = conv_tma_applies(g);
    if (fused) {
        g.head_w = n->P + kOffWh; g.head_b = n->P + kOffBh; g.head_out = n->out;
        if (!keep_pre) g.O = nullptr;
    }
    ISG_TRY_N(launch_gemm_bf16(g, s));
    if (!fused) k_head_fwd<<<(int)((R2 + 127) / 128), 128, 0, s>>>(n->H3, R2, n->P, n->out);
    if (cudaGetLastError() != cudaSuccess) return cuda_fail(cudaGetLastError(), "network forward");
    return ISING_OK;
}

// gradients of the mean NLL into G (zeroed here); windows/targets FP32 device arrays
int net_backward(ising_net* n, const float* win, const float* tgt, int nb) {
    cudaStream_t s = n->stream;
    const int64_t R1 = (int64_t)nb * 216, R2 = (int64_t)nb * 64;
    const int64_t L1 = (int64_t)pad32(R1), L2 = (int64_t)pad32(R2);
    ISG_CUDA(cudaMemsetAsync(n->G, 0, kNParams * sizeof(float), s));
    ISG_CUDA(cudaMemsetAsync(n->loss, 0, sizeof(double), s));
    k_nll<<<(int)((R2 + 127) / 128), 128, 0, s>>>(win, tgt, n->out, R2, 1.f / (float)R2, n->dout, n->loss);
    k_head_bwd<<<(int)((R2 + 127) / 128), 128, 0, s>>>(n->dout, n->H3, R2, n->P, n->dh, n->G);
    // conv3
    k_gelu_bwd<<<grid_for(kCh * L2), 256, 0, s>>>(n->dh, n->pre3, R2, L2, n->dp, n->dpt, n->G + kOffB3);
    k_im2col<<<grid_for((int64_t)kK2Pad * L2), 256, 0, s>>>(n->H2, kCh, 4, 4, 1, R2, n->AT, kK2, 1, L2, kK2Pad);
    GemmArgs g = gemm(n->AT, (int)L2, n->dpt, (int)L2, kK2, kCh, (int)L2, n->status);
    g.C = n->Cw; g.ldc = kCh;
    ISG_TRY_N(launch_gemm_bf16(g, s));
    k_scatter_wgrad<<<(27 * kCh * kCh + 255) / 256, 256, 0, s>>>(n->Cw, kCh, kCh, kOffW3, n->G);
    g = conv_gemm(n->dp, kCh, 4, 4, 1, n->W3fT, kK2, (int)R2, n->status);
    g.C = n->dh; g.ldc = kCh;
    ISG_TRY_N(launch_gemm_bf16(g, s));
    // conv2
    k_gelu_bwd<<<grid_for(kCh * L2), 256, 0, s>>>(n->dh, n->pre2, R2, L2, n->dp, n->dpt, n->G + kOffB2);
    k_im2col<<<grid_for((int64_t)kK2Pad * L2), 256, 0, s>>>(n->H1, kCh, 6, 4, 0, R2, n->AT, kK2, 1, L2, kK2Pad);
    g = gemm(n->AT, (int)L2, n->dpt, (int)L2, kK2, kCh, (int)L2, n->status);
    g.C = n->Cw; g.ldc = kCh;
    ISG_TRY_N(launch_gemm_bf16(g, s));
    k_scatter_wgrad<<<(27 * kCh * kCh + 255) / 256, 256, 0, s>>>(n->Cw, kCh, kCh, kOffW2, n->G);
    g = conv_gemm(n->dp, kCh, 4, 6, 2, n->W2fT, kK2, (int)R1, n->status);
    g.C = n->dh; g.ldc = kCh;
    ISG_TRY_N(launch_gemm_bf16(g, s));
    // conv1
    k_gelu_bwd<<<grid_for(kCh * L1), 256, 0, s>>>(n->dh, n->pre1, R1, L1, n->dp, n->dpt, n->G + kOffB1);
    k_im2col<<<grid_for((int64_t)256 * L1), 256, 0, s>>>(n->X0, kC0, 8, 6, 0, R1, n->AT, kK1, 1, L1, 256);
    g = gemm(n->AT, (int)L1, n->dpt, (int)L1, 27 * kC0, kCh, (int)L1, n->status);
    g.C = n->Cw; g.ldc = kCh;
    ISG_TRY_N(launch_gemm_bf16(g, s));
    k_scatter_wgrad<<<(27 * 3 * kCh + 255) / 256, 256, 0, s>>>(n->Cw, 3, kC0, kOffW1, n->G);
    if (cudaGetLastError() != cudaSuccess) return cuda_fail(cudaGetLastError(), "network backward");
    return ISING_OK;
}

int net_pack(ising_net* n) {
    k_pack<<<(kCh * kK2 + 255) / 256, 256, 0, n->stream>>>(n->P, n->Wf1, n->Wf2, n->Wf3, n->W2fT, n->W3fT);
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}

int net_check_batch(const ising_net* n, int nb) {
    if (nb < 1 || nb > n->max_batch) return fail(ISING_ERR_ARG, "batch must be 1..max_batch");
    return ISING_OK;
}

}  // namespace

extern "C" int ising_net_create(int device, int max_batch, uint64_t seed, ising_net** out) {
    if (!out) return fail(ISING_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (max_batch < 2 || max_batch > (1 << 16)) return fail(ISING_ERR_ARG, "max_batch must be 2..65536");
    max_batch += max_batch & 1;   // even batches keep every row count a multiple of 16
    NetGuard guard(device);
    std::unique_ptr<ising_net> n(new ising_net());
    n->device = device;
    n->max_batch = max_batch;
    auto bail = [&](int st) { net_free(n.get()); return st; };
    if (cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(cuda_fail(cudaGetLastError(), "cudaStreamCreateWithFlags"));
    const size_t B = (size_t)max_batch, R1 = B * 216, R2 = B * 64;
    const size_t L1 = pad32(R1);
    int st = ISING_OK;
    if ((st = nalloc(&n->P, kNParams)) || (st = nalloc(&n->G, kNParams)) || (st = nalloc(&n->M, kNParams)) ||
        (st = nalloc(&n->V, kNParams)) || (st = nalloc(&n->Wf1, kCh * kK1)) || (st = nalloc(&n->Wf2, kCh * kK2)) ||
        (st = nalloc(&n->Wf3, kCh * kK2)) || (st = nalloc(&n->W2fT, kCh * kK2)) || (st = nalloc(&n->W3fT, kCh * kK2)) ||
        (st = nalloc(&n->X0, B * 512 * kC0)) || (st = nalloc(&n->H1, R1 * kCh)) ||
        (st = nalloc(&n->H2, R2 * kCh)) ||
        (st = nalloc(&n->H3, R2 * kCh)) || (st = nalloc(&n->pre1, R1 * kCh)) || (st = nalloc(&n->pre2, R2 * kCh)) ||
        (st = nalloc(&n->pre3, R2 * kCh)) || (st = nalloc(&n->out, R2 * 4)) || (st = nalloc(&n->dout, R2 * 4)) ||
        (st = nalloc(&n->dh, R1 * kCh)) || (st = nalloc(&n->Cw, (size_t)kK2Pad * kCh)) ||
        (st = nalloc(&n->dp, R1 * kCh)) || (st = nalloc(&n->dpt, (size_t)kCh * L1)) ||
        (st = nalloc(&n->AT, std::max((size_t)kK2Pad * pad32(R2), (size_t)256 * L1))) ||
        (st = nalloc(&n->loss, 1)) || (st = nalloc(&n->status, 1)))
        return bail(st);
    // padding rows of the GEMM A operands stay zero
    cudaMemset(n->M, 0, kNParams * sizeof(float));
    cudaMemset(n->V, 0, kNParams * sizeof(float));
    cudaMemset(n->status, 0, sizeof(int));
    // He-normal convolutions, small head; log sigma bias log(0.3)
    std::vector<float> h(kNParams, 0.f);
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.f, 1.f);
    for (int i = 0; i < 2592; ++i) h[kOffW1 + i] = nd(rng) * std::sqrt(2.f / 81.f);
    for (int i = 0; i < 27648; ++i) h[kOffW2 + i] = nd(rng) * std::sqrt(2.f / 864.f);
    for (int i = 0; i < 27648; ++i) h[kOffW3 + i] = nd(rng) * std::sqrt(2.f / 864.f);
    for (int i = 0; i < 128; ++i) h[kOffWh + i] = nd(rng) * 0.01f;
    h[kOffBh + 3] = std::log(0.3f);
    if (cudaMemcpy(n->P, h.data(), kNParams * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(cuda_fail(cudaGetLastError(), "parameter upload"));
    if ((st = net_pack(n.get())) != ISING_OK) return bail(st);
    if (cudaStreamSynchronize(n->stream) != cudaSuccess) return bail(cuda_fail(cudaGetLastError(), "network init"));
    *out = n.release();
    return ISING_OK;
}

extern "C" int ising_net_destroy(ising_net* n) {
    if (!n) return ISING_OK;
    NetGuard guard(n->device);
    cudaStreamSynchronize(n->stream);
    net_free(n);
    delete n;
    return ISING_OK;
}

extern "C" int ising_net_param_count(void) { return kNParams; }

extern "C" int ising_net_set_params(ising_net* n, const float* host) {
    if (!n || !host) return fail(ISING_ERR_ARG, "NULL argument");
    NetGuard guard(n->device);
    ISG_CUDA(cudaMemcpyAsync(n->P, host, kNParams * sizeof(float), cudaMemcpyHostToDevice, n->stream));
    ISG_CUDA(cudaMemsetAsync(n->M, 0, kNParams * sizeof(float), n->stream));
    ISG_CUDA(cudaMemsetAsync(n->V, 0, kNParams * sizeof(float), n->stream));
    n->adam_t = 0;
    ISG_TRY(net_pack(n));
    ISG_CUDA(cudaStreamSynchronize(n->stream));
    return ISING_OK;
}

extern "C" int ising_net_get_params(const ising_net* n, float* host) {
    if (!n || !host) return fail(ISING_ERR_ARG, "NULL argument");
    NetGuard guard(n->device);
    ISG_CUDA(cudaMemcpyAsync(host, n->P, kNParams * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
    ISG_CUDA(cudaStreamSynchronize(n->stream));
    return ISING_OK;
}

extern "C" int ising_net_forward(ising_net* n, const float* d_windows, int nb, float* d_out) {
    if (!n || !d_windows || !d_out) return fail(ISING_ERR_ARG, "NULL argument");
    ISG_TRY(net_check_batch(n, nb));
    NetGuard guard(n->device);
    k_windows_to_rows<<<grid_for((int64_t)nb * 512), 256, 0, n->stream>>>(d_windows, nb, n->X0);
    ISG_TRY(net_forward_rows(n, nb, false));
    ISG_CUDA(cudaMemcpyAsync(d_out, n->out, (size_t)nb * 64 * 4 * sizeof(float), cudaMemcpyDeviceToDevice, n->stream));
    return net_check(n);
}

extern "C" int ising_net_loss_grad(ising_net* n, const float* d_windows, const float* d_targets, int nb, double* loss,
                                   float* host_grads) {
    if (!n || !d_windows || !d_targets) return fail(ISING_ERR_ARG, "NULL argument");
    ISG_TRY(net_check_batch(n, nb));
    NetGuard guard(n->device);
    k_windows_to_rows<<<grid_for((int64_t)nb * 512), 256, 0, n->stream>>>(d_windows, nb, n->X0);
    ISG_TRY(net_forward_rows(n, nb, true));
    ISG_TRY(net_backward(n, d_windows, d_targets, nb));
    double l = 0.0;
    ISG_CUDA(cudaMemcpyAsync(&l, n->loss, sizeof(double), cudaMemcpyDeviceToHost, n->stream));
    if (host_grads) ISG_CUDA(cudaMemcpyAsync(host_grads, n->G, kNParams * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
    ISG_TRY(net_check(n));
    if (loss) *loss = l / (double)((int64_t)nb * 64);
    return ISING_OK;
}

extern "C" int ising_net_train_step(ising_net* n, const float* d_windows, const float* d_targets, int nb, double lr,
                                    double* loss) {
    if (!n || !d_windows || !d_targets) return fail(ISING_ERR_ARG, "NULL argument");
    ISG_TRY(net_check_batch(n, nb));
    if (!(lr > 0.0) || !std::isfinite(lr)) return fail(ISING_ERR_ARG, "learning rate must be positive");
    NetGuard guard(n->device);
    k_windows_to_rows<<<grid_for((int64_t)nb * 512), 256, 0, n->stream>>>(d_windows, nb, n->X0);
    ISG_TRY(net_forward_rows(n, nb, true));
    ISG_TRY(net_backward(n, d_windows, d_targets, nb));
    ++n->adam_t;
    const float b1t = (float)std::pow(0.9, n->adam_t), b2t = (float)std::pow(0.999, n->adam_t);
    k_adam<<<(kNParams + 255) / 256, 256, 0, n->stream>>>(n->P, n->G, n->M, n->V, kNParams, (float)lr, b1t, b2t);
    ISG_TRY(net_pack(n));
    double l = 0.0;
    ISG_CUDA(cudaMemcpyAsync(&l, n->loss, sizeof(double), cudaMemcpyDeviceToHost, n->stream));
    ISG_TRY(net_check(n));
    if (loss) *loss = l / (double)((int64_t)nb * 64);
    return ISING_OK;
}

namespace isg {

__nv_bfloat16* net_rows(ising_net* n) { return n->X0; }
int net_forward_prepared(ising_net* n, int nb, cudaStream_t s, const float** out) {
    if (nb < 1 || nb > n->max_batch) return fail(ISING_ERR_ARG, "window batch exceeds the network's max_batch");
    cudaStream_t keep = n->stream;
    n->stream = s;
    const int st = net_forward_rows(n, nb, false);
    n->stream = keep;
    *out = n->out;
    return st;
}
int net_max_batch(const ising_net* n) { return n->max_batch; }
int net_status_on(ising_net* n, cudaStream_t s) {
    int h = 0;
    ISG_CUDA(cudaMemcpyAsync(&h, n->status, sizeof(int), cudaMemcpyDeviceToHost, s));
    ISG_CUDA(cudaStreamSynchronize(s));
    if (h) {
        cudaMemsetAsync(n->status, 0, sizeof(int), s);
        return fail(h & kStatTimeout ? ISING_ERR_TIMEOUT : ISING_ERR_NAN, "proposal network failed on the device");
    }
    return ISING_OK;
}
int net_device(const ising_net* n) { return n->device; }

}  // namespace isg
