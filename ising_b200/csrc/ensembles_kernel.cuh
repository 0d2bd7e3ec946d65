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

// ---- staged loader ------------------------------------------------------------------
__device__ __forceinline__ uint32_t st_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void st_tma5(const float* dst, const CUtensorMap* map, int c1, int c2, int c3, int c4,
                                        uint64_t* bar) {
    // innermost coordinate 0: every copy starts on a row boundary (256 bytes)
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(st_smem(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(st_smem(bar))
        : "memory");
}
__device__ __forceinline__ bool st_try(uint64_t* bar, uint32_t par) {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(st_smem(bar)), "r"(par) : "memory");
    return ok != 0;
}
// try_wait that may suspend the thread in hardware for up to 20 us while the phase is open
__device__ __forceinline__ bool st_try_suspend(uint64_t* bar, uint32_t par) {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(st_smem(bar)), "r"(par), "r"(20000u) : "memory");
    return ok != 0;
}
// bounded wait for phase parity `par`; gives up when the block's abort flag is raised or
// the wait passes the engine's bound (then raises the flags itself).  The poll count is a
// second bound in case the timer does not advance: a poll lasts from tens of nanoseconds
// to the 20 us suspend, so wait_ns / 4096 polls end within ~wait_ns / 100 .. 5 wait_ns.
static __device__ __forceinline__ bool st_wait(const EnsParams& P, uint64_t* bar, uint32_t par,
                                               volatile int* s_abort) {
    if (st_try(bar, par)) return true;
    const uint64_t t0 = global_ns();
    const uint64_t max_polls = P.wait_ns / 4096u + 4096u;
    for (uint64_t it = 0; it < max_polls; ++it) {
        if (st_try_suspend(bar, par)) return true;
        if (*s_abort) return false;
        if ((it & 63u) == 63u && global_ns() - t0 > P.wait_ns) break;
    }
    *s_abort = 1;
    atomicOr(P.status, kStatTimeout);
    atomicExch(P.abort, 1u);
    return false;
}

struct StRing {
    float* stages;     // this sub-block's kStStages stages
    uint64_t* full;    // [kStStages]: TMA transaction barriers
    uint64_t* empty;   // [kStStages]: one arrival per warp of the sub-block
    uint32_t cons;     // stages waited for so far (the same in every thread of the sub-block)
};

// Geometry of unit u of a task: plane group x0 .. x0+kStG-1, rows [ya, yb).
struct StUnit { uint32_t x0, ya, yb; };
__device__ __forceinline__ StUnit st_unit(const EnsDev& E, uint32_t x0c, uint32_t u) {
    const uint32_t grp = u / E.st_nseg, seg = u - grp * E.st_nseg;
    const uint32_t ya = seg * E.st_seg_len;
    return {x0c + grp * (uint32_t)kStG, ya, min(ya + E.st_seg_len, (uint32_t)E.g.ny)};
}

// Issue the copies of step t of unit U (stage sequence number n): the other colour's row
// ya + t - 1 (cyclic) of planes x0-1 .. x0+kStG and, for t >= 2, the own colour's row
// ya + t - 2 of planes x0 .. x0+kStG-1.
static __device__ __forceinline__ void st_issue(const EnsMaps& M, const EnsDev& E, const StRing& R, uint32_t n,
                                                const StUnit& U, uint32_t t, int colour, uint32_t rep) {
    const int nx = E.g.nx, ny = E.g.ny;
    const uint32_t slot = n % kStStages;
    float* st = R.stages + slot * kStStageFloats;
    uint64_t* fb = R.full + slot;
    int yn = (int)U.ya + (int)t - 1;
    yn = yn < 0 ? yn + ny : (yn >= ny ? yn - ny : yn);
    const uint32_t bytes = 4u * (t >= 2 ? kStStageFloats : kStNxtFloats);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(st_smem(fb)), "r"(bytes) : "memory");
    const int oc = colour ^ 1, c4 = 3 * (int)rep, x0 = (int)U.x0;
    if (x0 >= 1 && x0 + kStG < nx) {
        st_tma5(st, &M.next, yn, x0 - 1, oc, c4, fb);
    } else {   // the x-halo wraps: per component the centre planes and the two halo planes
        const int xm = x0 == 0 ? nx - 1 : x0 - 1, xp = x0 + kStG == nx ? 0 : x0 + kStG;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float* sc = st + c * (kStG + 2) * 64;
            st_tma5(sc, &M.halo, yn, xm, oc, c4 + c, fb);
            st_tma5(sc + 64, &M.ctr, yn, x0, oc, c4 + c, fb);
            st_tma5(sc + (kStG + 1) * 64, &M.halo, yn, xp, oc, c4 + c, fb);
        }
    }
    if (t >= 2) st_tma5(st + kStNxtFloats, &M.own, (int)(U.ya + t - 2), x0, colour, c4, fb);
}

// One task's colour pass with TMA-staged rows.  Warp g of sub-block sb (compute warps
// 0 .. kStSub * kStG - 1) updates plane x0 + g of units sb, sb + kStSub, ...; lane l the entry
// pair (2l, 2l+1).  The last warp issues the copies: its lane sb fills sub-block sb's ring as
// far as released stages allow.  False if a wait gave up (the copy lanes have then waited,
// boundedly, for the copies still in flight).
template <int MOVE, int DMI, bool HAS_K, int EI>
__device__ __forceinline__ bool run_chunk_staged(const EnsParams& P, uint32_t rep, uint32_t ph, uint32_t ch,
                                                 StRing& R, volatile int* s_abort, v2& de, v2& dmx, v2& dmy,
                                                 v2& dmz) {
    const EnsDev& E = P.e[EI];
    const CbGeom& G = E.g;
    const int colour = (int)(ph & 1u);
    const uint32_t ny = (uint32_t)G.ny, nx = (uint32_t)G.nx, xs = G.row_stride_x;
    const uint32_t x0c = ch * E.P;
    const uint32_t np = min(x0c + E.P, nx) - x0c;
    const uint32_t nunits = (np / (uint32_t)kStG) * E.st_nseg;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    bool ok = true;
    if (warp == (uint32_t)(kStSub * kStG)) {   // the copy warp
        if (lane >= (uint32_t)kStSub) return true;
        const EnsMaps& M = P.maps[EI];
        // the spins the copies read were published by st.release and acquired by this thread
        // in the generic proxy: order them before this task's async-proxy (TMA) reads
        asm volatile("fence.proxy.async.global;" ::: "memory");
        uint32_t m = R.cons;   // copy lanes: stages issued so far
#pragma unroll 1
        for (uint32_t u = lane; u < nunits && ok; u += kStSub) {
            const StUnit U = st_unit(E, x0c, u);
            const uint32_t T = U.yb - U.ya + 2u;
#pragma unroll 1
            for (uint32_t t = 0; t < T; ++t) {
                if (m >= (uint32_t)kStStages)
                    ok = st_wait(P, R.empty + m % kStStages, ((m / kStStages) - 1u) & 1u, s_abort);
                if (!ok) break;
                st_issue(M, E, R, m, U, t, colour, rep);
                ++m;
            }
        }
        if (!ok) {
            // the last kStStages stages issued may still write into the ring: let them land
            for (uint32_t q = m > (uint32_t)kStStages ? m - kStStages : 0u; q < m; ++q)
                for (uint32_t it = 0; it < (1u << 20); ++it)
                    if (st_try(R.full + q % kStStages, (q / kStStages) & 1u)) break;
        }
        R.cons = m;
        return ok;
    }
    const uint32_t sweep = __ldcg(E.sweep_ctr + rep) + (ph >> 1);
    const float beta2 = (float)(__ldcg(E.beta_rep + rep) * 1.4426950408889634);
    float* __restrict__ sx = E.spins + (size_t)rep * 3 * E.N;
    float* __restrict__ sy = sx + E.N;
    float* __restrict__ sz = sy + E.N;
    const uint32_t own = (uint32_t)colour * G.half;
    const uint32_t sb = warp / (uint32_t)kStG, g = warp - sb * (uint32_t)kStG;
    const uint32_t j = 2u * lane;
#pragma unroll 1
    for (uint32_t u = sb; u < nunits && ok; u += kStSub) {
        const StUnit U = st_unit(E, x0c, u);
        const uint32_t T = U.yb - U.ya + 2u;
        const uint32_t x = U.x0 + g;
#pragma unroll 1
        for (uint32_t t = 0; t < T; ++t) {
            const uint32_t n = R.cons;
            ok = st_wait(P, R.full + n % kStStages, (n / kStStages) & 1u, s_abort);
            if (!ok) break;
            R.cons = n + 1u;
            if (t < 2) continue;
            const uint32_t y = U.ya + t - 2u;
            const float* b0 = R.stages + (n % kStStages) * kStStageFloats;
            const float* b1 = R.stages + ((n - 1u) % kStStages) * kStStageFloats;
            const float* b2 = R.stages + ((n - 2u) % kStStages) * kStStageFloats;
            constexpr uint32_t cs = (kStG + 2) * 64;   // component stride of an other-colour stage
            const uint32_t o = (g + 1u) * 64u + j;
            auto l2 = [](const float* b, uint32_t off) { return *reinterpret_cast<const v2*>(b + off); };
            const float* bo = b0 + kStNxtFloats + g * 64u + j;
            const v23 s = {l2(bo, 0), l2(bo, kStG * 64), l2(bo, 2 * kStG * 64)};
            const v23 nxt = {l2(b0, o), l2(b0, cs + o), l2(b0, 2 * cs + o)};
            const v23 cur = {l2(b1, o), l2(b1, cs + o), l2(b1, 2 * cs + o)};
            const v23 prv = {l2(b2, o), l2(b2, cs + o), l2(b2, 2 * cs + o)};
            const v23 px = {l2(b1, o + 64), l2(b1, cs + o + 64), l2(b1, 2 * cs + o + 64)};
            const v23 mx = {l2(b1, o - 64), l2(b1, cs + o - 64), l2(b1, 2 * cs + o - 64)};
            const uint32_t p = (x + y + (uint32_t)colour) & 1u;
            const uint32_t je = p ? (j + 2u == 64u ? 0u : j + 2u) : (j == 0u ? 63u : j - 1u);
            const float* be = b1 + (g + 1u) * 64u + je;
            const float ex = be[0], ey = be[cs], ez = be[2 * cs];
            pair_compute<MOVE, DMI, HAS_K>(G, P.rk, P.status, sx, sy, sz, own + x * xs + y * 64u + j, x * ny + y, j,
                                           p, s, px, mx, nxt, prv, cur, ex, ey, ez, sweep, rep, beta2, de, dmx, dmy,
                                           dmz);
            // stage n-2 is no longer read; after the unit's last row neither are n-1 and n
            __syncwarp();
            if (lane == 0) {
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(st_smem(R.empty + (n - 2u) % kStStages))
                             : "memory");
                if (t + 1u == T) {
                    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(st_smem(R.empty + (n - 1u) % kStStages))
                                 : "memory");
                    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(st_smem(R.empty + n % kStStages))
                                 : "memory");
                }
            }
        }
    }
    return ok;
}

template <int MOVE, int DMI, bool HAS_K, bool STAGED>
__global__ void __launch_bounds__(STAGED ? kStThreads : kEnsMaxThreads, 2) k_ensembles(const __grid_constant__ EnsParams P) {
    __shared__ uint32_t s_task[5];
    __shared__ int s_go, s_fin;
    __shared__ volatile int s_abort;
    __shared__ float red[4][(kStThreads + 31) / 32];
    extern __shared__ __align__(128) unsigned char st_raw[];
    const uint32_t nph = 2u * P.k;
    const uint32_t tpr = P.tasks_per_round;
    const uint32_t total = tpr * P.rounds;
    StRing ring{};
    if (STAGED) {
        unsigned char* base = st_raw + ((128u - (st_smem(st_raw) & 127u)) & 127u);
        // compute warps by sub-block; lane sb of the copy warp serves sub-block sb
        const uint32_t w = threadIdx.x >> 5, l = threadIdx.x & 31u;
        const uint32_t sb = w < (uint32_t)(kStSub * kStG) ? w / (uint32_t)kStG : (l < (uint32_t)kStSub ? l : 0u);
        float* stages = reinterpret_cast<float*>(base);
        uint64_t* bars = reinterpret_cast<uint64_t*>(base + kStSub * kStStages * kStStageFloats * 4u);
        ring.stages = stages + sb * kStStages * kStStageFloats;
        ring.full = bars + sb * 2 * kStStages;
        ring.empty = ring.full + kStStages;
        ring.cons = 0;
        if (threadIdx.x == 0) {
            for (int i = 0; i < kStSub * kStStages; ++i) {
                asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(st_smem(bars + (i / kStStages) * 2 * kStStages + i % kStStages)), "r"(1));
                asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(st_smem(bars + (i / kStStages) * 2 * kStStages + kStStages + i % kStStages)), "r"(kStG));
            }
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
    }
    if (threadIdx.x == 0) s_abort = 0;
    __syncthreads();
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
        if (STAGED) {
            switch (e) {
#define ISG_EC(i) case i: run_chunk_staged<MOVE, DMI, HAS_K, i>(P, rep, ph, ch, ring, &s_abort, de, dmx, dmy, dmz); break;
                ISG_EC(0) ISG_EC(1) ISG_EC(2) ISG_EC(3) ISG_EC(4) ISG_EC(5) ISG_EC(6) ISG_EC(7)
                ISG_EC(8) ISG_EC(9) ISG_EC(10) ISG_EC(11) ISG_EC(12) ISG_EC(13) ISG_EC(14) ISG_EC(15)
#undef ISG_EC
                default: break;
            }
        } else {
            switch (e) {
#define ISG_EC(i) case i: run_chunk<MOVE, DMI, HAS_K, i>(P, rep, ph, ch, de, dmx, dmy, dmz); break;
                ISG_EC(0) ISG_EC(1) ISG_EC(2) ISG_EC(3) ISG_EC(4) ISG_EC(5) ISG_EC(6) ISG_EC(7)
                ISG_EC(8) ISG_EC(9) ISG_EC(10) ISG_EC(11) ISG_EC(12) ISG_EC(13) ISG_EC(14) ISG_EC(15)
#undef ISG_EC
                default: break;
            }
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
        if (STAGED && s_abort) break;   // a staged wait gave up: the chunk is incomplete
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
