// sweep_cb.cu -- checkerboard sweep over the colour-separated layout (simple cubic, even
// nx, ny and nz % 4 == 0), one launch per colour pass (or per paired pass of two replica
// groups).  The per-pair update is in sweep_cb.cuh.
//
// Per update this moves one read and one write of 12 bytes of its own colour plus 12 bytes
// of the other colour read as neighbours; a pass writes whole sectors only.
#include <algorithm>

#include "sweep_cb.cuh"

namespace isg {

#ifndef ISG_CB_MIN_BLOCKS
#define ISG_CB_MIN_BLOCKS 3
#endif
#ifndef ISG_CB_BLOCKS_PER_SM
#define ISG_CB_BLOCKS_PER_SM 3
#endif
constexpr int kCbThreads = 256;
constexpr int kNumSMs = 148;   // B200

struct CbParams {
    CbLaunch a;
    CbGeom g;
    FastDiv divNY;
    uint32_t W;             // packed row length nz/2
    uint32_t rows;          // packed rows per colour: nx * ny
    uint32_t rb;            // rows per block
    uint32_t step;          // rows advanced per loop iteration: gridDim.x * rb
    uint32_t step_x, step_y;// step = step_x * ny + step_y
    uint32_t rk[20];        // Philox round keys: key + i * (W0, W1), i = 0..9
};

template <int MOVE, int DMI, bool HAS_K>
__global__ void __launch_bounds__(kCbThreads, ISG_CB_MIN_BLOCKS) k_cb_sweep(const __grid_constant__ CbParams P) {
    const CbLaunch& a = P.a;
    int zi = blockIdx.y, sg = 0;
    if (zi >= a.seg[0].n_rep) { zi -= a.seg[0].n_rep; sg = 1; }
    const int colour = a.seg[sg].colour;
    const uint32_t rep = (uint32_t)(a.seg[sg].rep_first + zi);
    const int64_t N = a.natoms;
    float* __restrict__ sx = a.spins + (int64_t)rep * 3 * N;
    float* __restrict__ sy = sx + N;
    float* __restrict__ sz = sy + N;
    const uint32_t sweep = a.sweep_ctr[rep] + a.seg[sg].sweep_offset;
    const float beta2 = (float)(a.beta_rep[rep] * 1.4426950408889634);
    v2 de = V(0.f), dmx = V(0.f), dmy = V(0.f), dmz = V(0.f);
    // thread (tx, ty) owns entries j = 2 tx, 2 tx + 1 of rows ty + blockIdx.x*RB + k*step;
    // the block is whole warps, threads past RB rows only join the reduction
    const uint32_t tx = threadIdx.x % (P.W / 2u), ty = threadIdx.x / (P.W / 2u);
    const uint32_t j = 2u * tx;
    uint32_t row = ty < P.rb ? blockIdx.x * P.rb + ty : P.rows;
    uint32_t x = fdiv(row, P.divNY);
    uint32_t y = row - x * (uint32_t)a.ny;
#pragma unroll 1
    for (; row < P.rows; row += P.step) {
        pair_update<MOVE, DMI, HAS_K>(P.g, P.rk, a.status, sx, sy, sz, row, x, y, j, colour, sweep, rep, beta2, de, dmx, dmy, dmz);
        x += P.step_x;
        y += P.step_y;
        if (y >= (uint32_t)a.ny) { y -= (uint32_t)a.ny; ++x; }
    }
    if (a.partials) {
        __shared__ double tot[4];
        __shared__ float red[4][kCbThreads / 32];
        const int tid = threadIdx.x;
        const int lane = tid & 31, w = tid >> 5;
        float v0 = warp_sum(de.x + de.y), v1 = warp_sum(dmx.x + dmx.y);
        float v2_ = warp_sum(dmy.x + dmy.y), v3 = warp_sum(dmz.x + dmz.y);
        const int nw = (blockDim.x + 31) >> 5;
        if (lane == 0) { red[0][w] = v0; red[1][w] = v1; red[2][w] = v2_; red[3][w] = v3; }
        __syncthreads();
        if (tid < 4) {
            double t = 0.0;
            for (int k = 0; k < nw; ++k) t += (double)red[tid][k];
            tot[tid] = t;
            a.partials[((int64_t)rep * a.slots_per_rep + blockIdx.x) * 4 + tid] += t;
        }
    }
}

int cb_slots_per_rep() { return kNumSMs * ISG_CB_BLOCKS_PER_SM; }

template <int MOVE, int DMI>
static void cb_dispatch_k(const CbParams& P, dim3 g, dim3 b, bool hk, cudaStream_t s) {
    if (hk) k_cb_sweep<MOVE, DMI, true><<<g, b, 0, s>>>(P);
    else k_cb_sweep<MOVE, DMI, false><<<g, b, 0, s>>>(P);
}

int launch_cb_sweep(const CbLaunch& a, int move, int dmi, cudaStream_t s) {
    const int nrep = a.seg[0].n_rep + (a.n_seg > 1 ? a.seg[1].n_rep : 0);
    if (nrep <= 0) return ISING_OK;
    if (a.nz % 4 || a.nx % 2 || a.ny % 2) return fail(ISING_ERR_ARG, "colour-separated sweep needs even nx, ny and nz % 4 == 0");
    CbParams P;
    P.a = a;
    P.W = (uint32_t)(a.nz / 2);
    P.divNY = make_div((uint32_t)a.ny);
    P.rows = (uint32_t)(a.nx * a.ny);
    P.g.ham = a.ham;
    P.g.nx = a.nx; P.g.ny = a.ny; P.g.nz = a.nz;
    P.g.W = P.W;
    P.g.half = (uint32_t)(a.natoms / 2);
    P.g.row_stride_x = P.W * (uint32_t)a.ny;
    P.g.ensemble = a.ensemble;
    P.g.r = a.r;
    {
        philox_round_keys(a.seed, P.rk);
    }
    // block = (W/2 pair lanes) x (rows per block); about ISG_CB_BLOCKS_PER_SM resident blocks
    // per SM across the launch, at least one per replica
    const int tx = (int)(P.W / 2);
    if (tx > kCbThreads) return fail(ISING_ERR_ARG, "nz too large for the colour-separated sweep");
    const int ty = std::max(1, kCbThreads / tx);
    int zb = (kNumSMs * ISG_CB_BLOCKS_PER_SM + nrep - 1) / nrep;
    const int need = (int)((P.rows + ty - 1) / ty);
    if (zb > need) zb = need;
    if (zb > cb_slots_per_rep()) zb = cb_slots_per_rep();
    if (zb < 1) zb = 1;
    P.rb = (uint32_t)ty;
    P.step = (uint32_t)zb * (uint32_t)ty;
    P.step_x = P.step / (uint32_t)a.ny;
    P.step_y = P.step % (uint32_t)a.ny;
    dim3 g(zb, nrep), b(((tx * ty + 31) / 32) * 32);
    const bool hk = a.ham.K != 0.f;
#define ISG_CB(M, D) cb_dispatch_k<M, D>(P, g, b, hk, s)
    if (move == 0) {
        switch (dmi) { case 0: ISG_CB(0, 0); break; case 1: ISG_CB(0, 1); break;
                       case 2: ISG_CB(0, 2); break; default: ISG_CB(0, 3); }
    } else {
        switch (dmi) { case 0: ISG_CB(1, 0); break; case 1: ISG_CB(1, 1); break;
                       case 2: ISG_CB(1, 2); break; default: ISG_CB(1, 3); }
    }
#undef ISG_CB
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}

}  // namespace isg
