// ensembles_fused.cuh -- the persistent engine with both colour passes of a sweep fused into
// one pass over memory (temporal blocking along y).
//
// A task is (ensemble, replica, sweep, unit); a unit is a chunk of whole x-planes [x0, x1)
// times a y-segment [ya, yb).  Sweep s reads the replica's spins from one buffer and writes
// them, both colours, into the other (ping-pong; an even number of sweeps per round leaves
// every round's result in the mesh's own buffer), so the input of a sweep is never modified
// while it runs.  The block holds one thread row per x-plane of the chunk plus one halo plane
// on either side (threads = planes x W/2 pairs) and marches y: at step t it updates colour 0
// of row yc = ya - 1 + t and then colour 1 of row yc - 1, whose six colour-0 neighbours are
// final by then.  The halo planes and the rows ya - 1 and yb are updated as well but not
// written: with the same Philox key and the same inputs they reproduce bit for bit what the
// neighbouring task writes, so the colour-1 updates at the chunk's faces see the new colour-0
// values without waiting for that task.  The result is bit-identical to two separate colour
// passes (ensembles_kernel.cuh, sweep_cb.cu).
//
// Per step a thread loads one colour-0 and one colour-1 pair row (both one step ahead) and
// stores two; the x-neighbour rows of both colours come from the neighbouring thread rows
// through shared memory (three rotating row slots).  One mbarrier phase per step: a thread
// arrives once its new colour-0 row is in shared memory, draws the Philox numbers of its
// colour-1 pair (which need no neighbour data) and then waits, boundedly, for the others' rows.  DRAM moves 12 B
// read + 12 B written per site and sweep plus the halo planes' rows, against 36 B for two
// passes.
//
// Dependencies: a task of sweep s reads rows ya-2 .. yb+1 of planes x0-2 .. x1+1 of its input
// buffer (units of at least two planes and two rows keep that inside the neighbouring units)
// and writes its own unit of the other buffer, which the neighbouring units of sweep s-1 read.
// So it waits until the 3 x 3 neighbourhood of units (cyclic) has finished sweep s-1, which
// covers both the data it reads and the readers of what it overwrites.
#pragma once
#include "ensembles_kernel.cuh"

namespace isg {

__device__ __forceinline__ void st3(float* b, uint32_t N, uint32_t o, const v23& v) {
    *reinterpret_cast<v2*>(b + o) = v.x;
    *reinterpret_cast<v2*>(b + N + o) = v.y;
    *reinterpret_cast<v2*>(b + 2 * N + o) = v.z;
}
// a pair row in shared memory: [3][W] floats
__device__ __forceinline__ void sm_put(float* r, uint32_t W, uint32_t j, const v23& v) {
    *reinterpret_cast<v2*>(r + j) = v.x;
    *reinterpret_cast<v2*>(r + W + j) = v.y;
    *reinterpret_cast<v2*>(r + 2 * W + j) = v.z;
}
__device__ __forceinline__ v23 sm_get(const float* r, uint32_t W, uint32_t j) {
    return {*reinterpret_cast<const v2*>(r + j), *reinterpret_cast<const v2*>(r + W + j),
            *reinterpret_cast<const v2*>(r + 2 * W + j)};
}

// Shared memory of a fused task: colour-1 (old) rows [3][np + 2][3][W] (slot 0 and np + 1 are
// the planes outside the halo planes), then colour-0 (new) rows [3][np][3][W]; three row
// slots rotate with y, so rows yc - 1, yc (and yc + 1 being written) coexist.
__host__ __device__ __forceinline__ uint32_t fused_smem_floats(uint32_t np, uint32_t W) {
    return (3u * (np + 2u) + 3u * np) * 3u * W;
}

// One fused task: sweep `sw` of the round (input buffer by its parity) over unit `u` of
// replica `rep`.
template <int MOVE, int DMI, bool HAS_K, int EI>
__device__ __forceinline__ void run_fused(const EnsParams& P, uint32_t rep, uint32_t sw, uint32_t u, float* sm,
                                          uint64_t* bar, uint32_t& bphase, volatile int* s_abort, v2& de, v2& dmx,
                                          v2& dmy, v2& dmz) {
    const EnsDev& E = P.e[EI];
    const CbGeom& G = E.g;
    const uint32_t nx = (uint32_t)G.nx, ny = (uint32_t)G.ny, W = G.W, xs = G.row_stride_x, half = G.half, N = E.N;
    const uint32_t ch = u / E.fnseg, sg = u - ch * E.fnseg;
    const uint32_t x0 = ch * nx / E.fnch, x1 = (ch + 1u) * nx / E.fnch;
    const uint32_t ya = sg * ny / E.fnseg, yb = (sg + 1u) * ny / E.fnseg;
    const uint32_t npe = x1 - x0 + 2u, Y = yb - ya, T = Y + 2u;
    const uint32_t sweep = __ldcg(E.sweep_ctr + rep) + sw;
    const float beta2 = (float)(__ldcg(E.beta_rep + rep) * 1.4426950408889634);
    const size_t roff = (size_t)rep * 3u * N;
    const float* in = ((sw & 1u) ? E.spins_b : E.spins) + roff;
    float* out = ((sw & 1u) ? E.spins : E.spins_b) + roff;
    const uint32_t i = fdiv(threadIdx.x, E.divTX), j = 2u * (threadIdx.x - i * E.divTX.d);
    const bool active = i < npe;
    const bool halo = i == 0u || i + 1u == npe;
    int xi = (int)x0 - 1 + (int)i;
    xi = xi < 0 ? xi + (int)nx : (xi >= (int)nx ? xi - (int)nx : xi);
    const uint32_t x = (uint32_t)xi;
    int xoi = i == 0u ? xi - 1 : xi + 1;   // halo planes: the plane outside
    xoi = xoi < 0 ? xoi + (int)nx : (xoi >= (int)nx ? xoi - (int)nx : xoi);
    const uint32_t xo = (uint32_t)xoi;
    const uint32_t np = E.fnp;
    const uint32_t rowf = 3u * W;
    const uint32_t kslab = (np + 2u) * rowf, wslab = np * rowf;
    float* ksm = sm + (i + 1u) * rowf;                // colour 1 (old), this plane's row in slot 0
    float* wsm = sm + 3u * kslab + i * rowf;          // colour 0 (new), this plane's row in slot 0
    const uint32_t oslot = i == 0u ? 0u : npe + 1u;   // where a halo row puts the outside plane
    float* osm = sm + oslot * rowf;
    auto up = [ny](uint32_t y) { return y + 1u == ny ? 0u : y + 1u; };
    auto dn = [ny](uint32_t y) { return y == 0u ? ny - 1u : y - 1u; };
    const float* ix = in;
    const float* iy = in + N;
    const float* iz = in + 2u * N;
    auto ldK = [&](uint32_t xp, uint32_t y) { return ld3(ix, iy, iz, half + xp * xs + y * W + j); };
    auto ldW = [&](uint32_t xp, uint32_t y) { return ld3(ix, iy, iz, xp * xs + y * W + j); };

    // row slots: s0 holds row yc, s2 row yc - 1, s1 row yc - 2 (colour 0) and receives row
    // yc + 1 (colour 1)
    uint32_t yc = ya == 0u ? ny - 1u : ya - 1u;
    uint32_t s0 = 0u, s1 = 1u, s2 = 2u;
    v23 Kn{}, Wo{}, pfK{}, pfW{}, pfO{};
    if (active) {
        sm_put(ksm + 2u * kslab, W, j, ldK(x, dn(yc)));
        sm_put(ksm, W, j, ldK(x, yc));
        Kn = ldK(x, up(yc));
        Wo = ldW(x, yc);
        pfW = ldW(x, up(yc));
        pfK = ldK(x, up(up(yc)));
        if (halo) {
            sm_put(osm, W, j, ldK(xo, yc));
            pfO = ldK(xo, up(yc));
        }
    }
    __syncthreads();
#pragma unroll 1
    for (uint32_t t = 0; t < T; ++t) {
        const uint32_t ym = dn(yc);
        const uint32_t p1 = (x + ym + 1u) & 1u;
        v23 Wn{};
        if (active) {
            // colour 0 at row yc against the old colour-1 rows
            const float* kc = ksm + s0 * kslab;
            const uint32_t p0 = (x + yc) & 1u;
            const uint32_t je = p0 ? (j + 2u == W ? 0u : j + 2u) : (j == 0u ? W - 1u : j - 1u);
            const bool inrow = t >= 1u && t <= Y;
            bool any;
            Wn = pair_new<MOVE, DMI, HAS_K>(
                G, P.rk, P.status, x * ny + yc, j, p0, Wo, sm_get(kc + rowf, W, j), sm_get(kc - rowf, W, j), Kn,
                sm_get(ksm + s2 * kslab, W, j), sm_get(kc, W, j), kc[je], kc[W + je], kc[2u * W + je], sweep, rep,
                beta2, inrow && !halo, de, dmx, dmy, dmz, any);
            sm_put(wsm + s0 * wslab, W, j, Wn);
            if (!halo && inrow) st3(out, N, x * xs + yc * W + j, Wn);
            // the next step's colour-1 rows: row yc + 1 of this plane and of the outside plane
            sm_put(ksm + s1 * kslab, W, j, Kn);
            if (halo) sm_put(osm + s1 * kslab, W, j, pfO);
            // registers of the next step, and the loads of the step after it
            Kn = pfK;
            Wo = pfW;
            if (t + 2u < T) {
                const uint32_t y2 = up(up(yc));
                pfW = ldW(x, y2);
                pfK = ldK(x, up(y2));
                if (halo) pfO = ldK(xo, y2);
            }
        }
        // the new rows are published by the arrival on the step's mbarrier phase (release); the
        // colour-1 pair's Philox draws, which need none of them, fill the time until every
        // thread has arrived.  The wait is bounded (st_wait): one that gives up raises the
        // block's and the engine's abort flags, and every thread then leaves the march.
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(st_smem(bar)) : "memory");
        const bool c1 = active && !halo && t >= 2u;
        uint4 ra = make_uint4(0u, 0u, 0u, 0u), rb = ra;
        if (c1) pair_draws(G, P.rk, x * ny + ym, j, p1, sweep, rep, ra, rb);
        const bool ok = st_wait(P, bar, bphase & 1u, s_abort);
        ++bphase;
        if (!ok) break;
        if (c1) {
            // colour 1 at row yc - 1: its colour-0 neighbours are rows yc-2 .. yc of this plane
            // and row yc - 1 of planes x +- 1 (written last step)
            const float* wc = wsm + s2 * wslab;
            const uint32_t je1 = p1 ? (j + 2u == W ? 0u : j + 2u) : (j == 0u ? W - 1u : j - 1u);
            bool any;
            const v23 Kw = pair_new_drawn<MOVE, DMI, HAS_K>(
                G, P.status, p1, sm_get(ksm + s2 * kslab, W, j), sm_get(wc + rowf, W, j), sm_get(wc - rowf, W, j),
                Wn, sm_get(wsm + s1 * wslab, W, j), sm_get(wc, W, j), wc[je1], wc[W + je1], wc[2u * W + je1], ra, rb,
                beta2, true, de, dmx, dmy, dmz, any);
            st3(out, N, half + x * xs + ym * W + j, Kw);
        }
        {
            const uint32_t r = s0;
            s0 = s1; s1 = s2; s2 = r;
        }
        yc = up(yc);
    }
}

template <int MOVE, int DMI, bool HAS_K>
__global__ void __launch_bounds__(kFuMaxThreads, 1) k_ensembles_fused(const __grid_constant__ EnsParams P) {
    __shared__ uint32_t s_task[5];
    __shared__ int s_go, s_fin;
    __shared__ float red[4][kFuMaxThreads / 32];
    __shared__ __align__(8) uint64_t fu_bar;   // one phase per y-step, all threads arrive
    __shared__ volatile int fu_abort;
    extern __shared__ __align__(16) float fu_sm[];
    const uint32_t k = P.k;
    const uint32_t tpr = P.tasks_per_round;
    const uint32_t total = tpr * P.rounds;
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(st_smem(&fu_bar)), "r"(blockDim.x));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        fu_abort = 0;
    }
    __syncthreads();
    uint32_t bphase = 0;   // steps completed on fu_bar (the same count in every thread)
    uint32_t next = 0;
    if (threadIdx.x == 0) next = atomicAdd(P.head, 1u);
    for (;;) {
        if (threadIdx.x == 0) {
            int go = 0;
            const uint32_t id = next;
            if (id < total && !*(volatile const uint32_t*)P.abort) {
                const uint32_t q = id / tpr;
                const uint2 t = __ldg(P.table + (id - q * tpr));
                const uint32_t e = t.x >> 24, r = t.x & 0xffffffu, sw = t.y >> 16, u = t.y & 0xffffu;
                const EnsDev& E = P.e[e];
                const uint32_t phi = q * k + sw;
                const uint32_t* d = E.done + (size_t)r * E.nch;
                go = 1;
                if (sw == 0 && q > 0) go = wait_ge(P, E.ready, (int)e == P.stall_ens ? 0x40000000u : q, id);
                if (go && phi > 0) {
                    const uint32_t nc = E.fnch, ns = E.fnseg, ch = u / ns, sg = u - ch * ns;
#pragma unroll 1
                    for (int a = 0; a < 9 && go; ++a) {
                        const uint32_t c2 = (ch + nc + (uint32_t)(a / 3) - 1u) % nc;
                        const uint32_t s2 = (sg + ns + (uint32_t)(a % 3) - 1u) % ns;
                        go = wait_ge(P, d + c2 * ns + s2, phi, id);
                    }
                }
                s_task[0] = e; s_task[1] = r; s_task[2] = sw; s_task[3] = u; s_task[4] = q;
            }
            s_go = go;
        }
        __syncthreads();
        if (!s_go) break;
        if (threadIdx.x == 0) next = atomicAdd(P.head, 1u);   // prefetch; used next iteration
        const uint32_t e = s_task[0], rep = s_task[1], sw = s_task[2], u = s_task[3], q = s_task[4];
        const EnsDev& E = P.e[e];
        const uint32_t phi = q * k + sw;
        if (threadIdx.x != 0 && phi > 0) {
            // every thread acquires the counters thread 0 found final before reading spins
            const uint32_t* d = E.done + (size_t)rep * E.nch;
            const uint32_t nc = E.fnch, ns = E.fnseg, ch = u / ns, sg = u - ch * ns;
#pragma unroll 1
            for (int a = 0; a < 9; ++a)
                ld_acquire(d + ((ch + nc + (uint32_t)(a / 3) - 1u) % nc) * ns + (sg + ns + (uint32_t)(a % 3) - 1u) % ns);
            if (sw == 0 && q > 0) ld_acquire(E.ready);
        }
        v2 de = V(0.f), dmx = V(0.f), dmy = V(0.f), dmz = V(0.f);
        switch (e) {
#define ISG_EC(i) case i: run_fused<MOVE, DMI, HAS_K, i>(P, rep, sw, u, fu_sm, &fu_bar, bphase, &fu_abort, de, dmx, dmy, dmz); break;
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
                for (int kk = 0; kk < nw; ++kk) t += (double)red[tid][kk];
                double* p = E.partials + ((size_t)rep * E.nch + u) * 4 + tid;
                __stcg(p, __ldcg(p) + t);
            }
        }
        __syncthreads();
        if (fu_abort) break;   // a step's wait gave up: the unit is incomplete
        if (threadIdx.x == 0) {
            __threadfence();
            st_release(E.done + (size_t)rep * E.nch + u, phi + 1u);
            int fin = 0;
            if (sw == k - 1u) {
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
