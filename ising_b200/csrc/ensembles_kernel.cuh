// ensembles_kernel.cuh -- persistent kernel running every PT replica of many colour-separated
// simple-cubic ensembles (uneven sizes and Hamiltonians) from one task queue.
//
// Each block loops: take the next task id (prefetched one task ahead), wait until the
// task's inputs are final, update the task's chunk with the pair update of sweep_cb.cuh,
// add its dE / dM sums to the chunk's partial slot, and publish the chunk's phase count.
// The block that finishes the last task of a round of an ensemble folds that ensemble's
// partials into its FP64 accumulators, runs the exchange (exchange.cuh), advances the sweep
// counters and publishes the round.  Every wait is bounded in time; a wait that gives up
// sets kStatTimeout, records the task and raises the abort word, after which every block
// stops at its next wait or queue fetch.
//
// Memory ordering: a task publishes with __syncthreads, __threadfence and st.release.gpu
// of its counter; a waiting block observes counters with ld.acquire.gpu in thread 0 and then
// in every thread before the chunk's loads.  Partial sums, accumulators, betas and counters
// that different SMs write in turn are accessed with ld.global.cg / st.global.cg.
#pragma once
#include "ensembles.h"
#include "exchange.cuh"

namespace isg {

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Thread 0 only: wait until *p >= target.  False when the engine aborts or the wait runs
// past P.wait_ns (then the engine is aborted here).  The poll count is bounded as well, in
// case the timer does not advance.
static __device__ __forceinline__ bool wait_ge(const EnsParams& P, const uint32_t* p, uint32_t target, uint32_t task) {
    if (ld_acquire(p) >= target) return true;
    const uint64_t t0 = global_ns();
    const uint64_t max_polls = P.wait_ns / 32u + 1024u;
    uint32_t ns = 32;
    for (uint64_t it = 0; it < max_polls; ++it) {
        __nanosleep(ns);
        if (ns < 512) ns <<= 1;
        if (ld_acquire(p) >= target) return true;
        if (*(volatile const uint32_t*)P.abort) return false;
        if (global_ns() - t0 > P.wait_ns) break;
    }
    atomicOr(P.status, kStatTimeout);
    atomicCAS(P.where, 0u, task + 1u);
    atomicExch(P.abort, 1u);
    __threadfence();
    return false;
}

// Whole block: end of round q of ensemble E.
static __device__ __forceinline__ void finish_round(const EnsParams& P, const EnsDev& E) {
    const int nw = (int)(blockDim.x >> 5), w = (int)(threadIdx.x >> 5), lane = (int)(threadIdx.x & 31);
    for (int r = w; r < E.n_rep; r += nw) {
        double* p = E.partials + (size_t)r * E.nch * 4;
        double v0 = 0.0, v1 = 0.0, v2_ = 0.0, v3 = 0.0;
        for (uint32_t c = lane; c < E.nch; c += 32) {
            v0 += __ldcg(p + 4 * c); v1 += __ldcg(p + 4 * c + 1);
            v2_ += __ldcg(p + 4 * c + 2); v3 += __ldcg(p + 4 * c + 3);
            __stcg(p + 4 * c, 0.0); __stcg(p + 4 * c + 1, 0.0);
            __stcg(p + 4 * c + 2, 0.0); __stcg(p + 4 * c + 3, 0.0);
        }
        v0 = warp_sum(v0); v1 = warp_sum(v1); v2_ = warp_sum(v2_); v3 = warp_sum(v3);
        if (lane == 0) {
            Acc4* a = E.acc + r;
            __stcg(&a->e, __ldcg(&a->e) + v0);
            __stcg(&a->mx, __ldcg(&a->mx) + v1);
            __stcg(&a->my, __ldcg(&a->my) + v2_);
            __stcg(&a->mz, __ldcg(&a->mz) + v3);
        }
    }
    __syncthreads();
    if (E.n_rep >= 2) {
        ExchangeLaunch ex;
        ex.n = E.n_rep; ex.beta_t = E.beta_t; ex.beta_rep = E.beta_rep; ex.t2r = E.t2r; ex.r2t = E.r2t;
        ex.acc = E.acc; ex.stats = E.stats; ex.round = E.round_ctr; ex.seed = P.seed;
        ex.ensemble = E.g.ensemble; ex.scheme = P.scheme;
        exchange_round(ex);
    }
    for (int r = threadIdx.x; r < E.n_rep; r += blockDim.x) __stcg(E.sweep_ctr + r, __ldcg(E.sweep_ctr + r) + P.k);
}

// One task's colour pass over x-planes [x0, x1): columns (plane, y-segment), nseg segments
// per plane so that every thread row is busy, each marched along y (march_column).
template <int MOVE, int DMI, bool HAS_K, int EI>
__device__ __forceinline__ void run_chunk(const EnsParams& P, uint32_t rep, uint32_t ph, uint32_t ch,
                                          v2& de, v2& dmx, v2& dmy, v2& dmz) {
    const EnsDev& E = P.e[EI];
    const CbGeom& G = E.g;
    const int colour = (int)(ph & 1u);
    const uint32_t sweep = __ldcg(E.sweep_ctr + rep) + (ph >> 1);
    const float beta2 = (float)(__ldcg(E.beta_rep + rep) * 1.4426950408889634);
    float* __restrict__ sx = E.spins + (size_t)rep * 3 * E.N;
    float* __restrict__ sy = sx + E.N;
    float* __restrict__ sz = sy + E.N;
    const uint32_t ny = (uint32_t)G.ny, nx = (uint32_t)G.nx;
    const uint32_t x0 = ch * E.P;
    const uint32_t np = min(x0 + E.P, nx) - x0;
    const uint32_t ty = fdiv(threadIdx.x, E.divTX);
    const uint32_t j = 2u * (threadIdx.x - ty * E.divTX.d);
    if (ty >= E.rb) return;
#pragma unroll 1
    for (uint32_t col = ty; col < np * E.nseg; col += E.rb) {
        const uint32_t xo = fdiv(col, E.divSeg), seg = col - xo * E.nseg;
        const uint32_t x = x0 + xo;
        const uint32_t ya = seg * E.seg_len, yb = min(ya + E.seg_len, ny);
        if (ya >= yb) continue;
        march_column<MOVE, DMI, HAS_K>(G, P.rk, P.status, sx, sy, sz, x, ya, yb, j, colour, sweep, rep, beta2, de, dmx,
                                       dmy, dmz);
    }
}

template <int MOVE, int DMI, bool HAS_K>
__global__ void __launch_bounds__(kEnsMaxThreads, 2) k_ensembles(const __grid_constant__ EnsParams P) {
    __shared__ uint32_t s_task[5];
    __shared__ int s_go, s_fin;
    __shared__ float red[4][kEnsMaxThreads / 32];
    const uint32_t nph = 2u * P.k;
    const uint32_t tpr = P.tasks_per_round;
    const uint32_t total = tpr * P.rounds;
    uint32_t next = 0;
    if (threadIdx.x == 0) next = atomicAdd(P.head, 1u);
    for (;;) {
        if (threadIdx.x == 0) {
            int go = 0;
            const uint32_t id = next;
            if (id < total && !*(volatile const uint32_t*)P.abort) {
                const uint32_t q = id / tpr;
                const uint2 t = __ldg(P.table + (id - q * tpr));
                const uint32_t e = t.x >> 24, r = t.x & 0xffffffu, ph = t.y >> 16, ch = t.y & 0xffffu;
                const EnsDev& E = P.e[e];
                const uint32_t phi = q * nph + ph;
                const uint32_t* d = E.done + (size_t)r * E.nch;
                const uint32_t cm = ch == 0 ? E.nch - 1 : ch - 1, cp = ch + 1 == E.nch ? 0 : ch + 1;
                go = 1;
                if (ph == 0 && q > 0)
                    go = wait_ge(P, E.ready, (int)e == P.stall_ens ? 0x40000000u : q, id);
                if (go && phi > 0)
                    go = wait_ge(P, d + ch, phi, id) && wait_ge(P, d + cm, phi, id) && wait_ge(P, d + cp, phi, id);
                s_task[0] = e; s_task[1] = r; s_task[2] = ph; s_task[3] = ch; s_task[4] = q;
            }
            s_go = go;
        }
        __syncthreads();
        if (!s_go) break;
        if (threadIdx.x == 0) next = atomicAdd(P.head, 1u);   // prefetch; used next iteration
        const uint32_t e = s_task[0], rep = s_task[1], ph = s_task[2], ch = s_task[3], q = s_task[4];
        const EnsDev& E = P.e[e];
        const uint32_t phi = q * nph + ph;
        if (threadIdx.x != 0 && phi > 0) {
            // every thread acquires the counters thread 0 found final before reading spins
            const uint32_t* d = E.done + (size_t)rep * E.nch;
            const uint32_t cm = ch == 0 ? E.nch - 1 : ch - 1, cp = ch + 1 == E.nch ? 0 : ch + 1;
            ld_acquire(d + ch);
            ld_acquire(d + cm);
            ld_acquire(d + cp);
            if (ph == 0 && q > 0) ld_acquire(E.ready);
        }
        v2 de = V(0.f), dmx = V(0.f), dmy = V(0.f), dmz = V(0.f);
        switch (e) {
#define ISG_EC(i) case i: run_chunk<MOVE, DMI, HAS_K, i>(P, rep, ph, ch, de, dmx, dmy, dmz); break;
            ISG_EC(0) ISG_EC(1) ISG_EC(2) ISG_EC(3) ISG_EC(4) ISG_EC(5) ISG_EC(6) ISG_EC(7)
            ISG_EC(8) ISG_EC(9) ISG_EC(10) ISG_EC(11) ISG_EC(12) ISG_EC(13) ISG_EC(14) ISG_EC(15)
#undef ISG_EC
            default: break;
        }
        {
            const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
            const float v0 = warp_sum(de.x + de.y), v1 = warp_sum(dmx.x + dmx.y);
            const float v2_ = warp_sum(dmy.x + dmy.y), v3 = warp_sum(dmz.x + dmz.y);
            if (lane == 0) { red[0][w] = v0; red[1][w] = v1; red[2][w] = v2_; red[3][w] = v3; }
            __syncthreads();
            if (tid < 4) {
                const int nw = (int)(blockDim.x >> 5);
                double t = 0.0;
                for (int k = 0; k < nw; ++k) t += (double)red[tid][k];
                double* p = E.partials + ((size_t)rep * E.nch + ch) * 4 + tid;
                __stcg(p, __ldcg(p) + t);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            st_release(E.done + (size_t)rep * E.nch + ch, phi + 1u);
            int fin = 0;
            if (ph == nph - 1) {
                const unsigned long long c = atomicAdd(E.fin, 1ull) + 1ull;
                fin = c == (unsigned long long)(q + 1) * (unsigned long long)E.n_rep * E.nch;
            }
            s_fin = fin;
        }
        __syncthreads();
        if (s_fin) {
            __threadfence();
            finish_round(P, E);
            __syncthreads();
            if (threadIdx.x == 0) {
                __threadfence();
                st_release(E.ready, q + 1u);
            }
        }
    }
}

}  // namespace isg
