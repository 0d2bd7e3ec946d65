// sweep_tma.cu -- checkerboard colour pass with TMA-staged neighbour rows (sm_100a).
//
// Same arithmetic and storage as sweep_cb.cu (colour-separated layout, pairs of sites per
// thread in packed FP32x2), but a block owns a slab of RS consecutive packed rows
// (x, y0..y0+RS-1) and marches along x through a chunk of planes.  The rows it needs are
// brought into shared memory by bulk asynchronous copies (cp.async.bulk, completion counted
// on an mbarrier): for plane x+1 the other colour's rows y0-1..y0+RS (the y halo included)
// and for plane x its own rows.  A ring of stages keeps two planes in flight while plane x
// is computed, so the DRAM latency overlaps the arithmetic instead of stalling warps.
//
// Every mbarrier wait is bounded; a wait that gives up sets the timeout status bit, drains
// the copies still in flight (again bounded) and leaves the kernel.
#include <algorithm>

#include "internal.h"

namespace isg {

namespace {

constexpr int kTmaMaxThreads = 256;
constexpr int kOthStages = 5;     // other-colour planes: x-1, x, x+1 in use, x+2, x+3 in flight
constexpr int kOwnStages = 3;     // own-colour planes: x in use, x+1, x+2 in flight
constexpr uint32_t kWaitLimit = 1u << 22;   // ~0.1 s of polling; a healthy copy lands in microseconds

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// bounded wait for the phase `parity` of an mbarrier; false if it gave up
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < kWaitLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// shorter bounded wait used only to drain copies after a timeout
__device__ __forceinline__ void mbar_wait_drain(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < (1u << 20); ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return;
    }
}

using v2 = float2;
__device__ __forceinline__ v2 V(float a) { return make_float2(a, a); }
__device__ __forceinline__ v2 add(v2 a, v2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ v2 sub(v2 a, v2 b) { return __ffma2_rn(b, V(-1.f), a); }
__device__ __forceinline__ v2 mul(v2 a, v2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ v2 fma2(v2 a, v2 b, v2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ v2 u01x2(uint32_t a, uint32_t b) {
    return __fadd2_rn(make_float2(__uint_as_float((a >> 9) | 0x3f800000u), __uint_as_float((b >> 9) | 0x3f800000u)),
                      V(-0.99999994f));
}

struct v23 { v2 x, y, z; };

struct TmaParams {
    CbLaunch a;
    uint32_t W;          // packed row length nz/2
    uint32_t RS;         // rows per slab (a divisor of ny)
    uint32_t XC;         // planes per x chunk
    uint32_t nslab;      // ny / RS
    uint32_t nchunk;     // ceil(nx / XC)
    uint32_t half;       // N/2
    uint32_t rk[20];     // Philox round keys
};

template <int MOVE>
__device__ __forceinline__ v23 propose2(const v23& s, uint4 ra, uint4 rb, float r) {
    const v2 u0 = u01x2(ra.x, rb.x), u1 = u01x2(ra.y, rb.y);
    const v2 cz = fma2(V(2.f), u0, V(-1.f));
    const v2 q = fma2(make_float2(-cz.x, -cz.y), cz, V(1.f));
    const v2 ph = fma2(V(6.28318531f), u1, V(-3.14159265f));
    const v2 st = make_float2(ax_sqrt(q.x), ax_sqrt(q.y));
    v23 v = {mul(st, make_float2(ax_cos(ph.x), ax_cos(ph.y))), mul(st, make_float2(ax_sin(ph.x), ax_sin(ph.y))), cz};
    if (MOVE == 1) {
        const v2 u2 = u01x2(ra.z, rb.z);
        const v2 lg = mul(make_float2(ax_lg2(u2.x), ax_lg2(u2.y)), V(0.33333334f));
        const v2 rho = mul(V(r), make_float2(ax_ex2(lg.x), ax_ex2(lg.y)));
        v = {fma2(rho, v.x, s.x), fma2(rho, v.y, s.y), fma2(rho, v.z, s.z)};
        const v2 n2 = fma2(v.x, v.x, fma2(v.y, v.y, mul(v.z, v.z)));
        const v2 rn = make_float2(ax_rsqrt(n2.x), ax_rsqrt(n2.y));
        v = {mul(v.x, rn), mul(v.y, rn), mul(v.z, rn)};
    }
    return v;
}

}  // namespace

// Shared memory: other-colour stages [kOthStages][3][RS+2][W], own stages [kOwnStages][3][RS][W].
template <int MOVE, int DMI, bool HAS_K>
__global__ void __launch_bounds__(kTmaMaxThreads, 3) k_cb_tma(const __grid_constant__ TmaParams P) {
    extern __shared__ __align__(128) float sm[];
    __shared__ __align__(8) uint64_t bar_oth[kOthStages];
    __shared__ __align__(8) uint64_t bar_own[kOwnStages];
    __shared__ int abort_flag;
    const CbLaunch& a = P.a;
    const HamDev& H = a.ham;
    const uint32_t W = P.W, RS = P.RS;
    const uint32_t oth_plane = 3u * (RS + 2u) * W;   // floats per other-colour stage
    const uint32_t own_plane = 3u * RS * W;
    float* oth_s = sm;
    float* own_s = sm + kOthStages * oth_plane;

    // block -> (segment replica, colour, slab, x chunk)
    uint32_t bid = blockIdx.x;
    const uint32_t chunk = bid % P.nchunk; bid /= P.nchunk;
    const uint32_t slab = bid % P.nslab; bid /= P.nslab;
    int zi = (int)bid, sg = 0;
    if (zi >= a.seg[0].n_rep) { zi -= a.seg[0].n_rep; sg = 1; }
    const int colour = a.seg[sg].colour;
    const uint32_t rep = (uint32_t)(a.seg[sg].rep_first + zi);
    const int nx = a.nx, ny = a.ny;
    const int64_t N = a.natoms;
    float* __restrict__ gs = a.spins + (int64_t)rep * 3 * N;   // x plane; y at +N, z at +2N
    const uint32_t own_base = (uint32_t)colour * P.half, oth_base = (uint32_t)(colour ^ 1) * P.half;
    const uint32_t y0 = slab * RS;
    const int x0 = (int)(chunk * P.XC);
    const int x1 = min(x0 + (int)P.XC, nx);
    const uint32_t sweep = a.sweep_ctr[rep] + a.seg[sg].sweep_offset;
    const float beta2 = (float)(a.beta_rep[rep] * 1.4426950408889634);
    const uint32_t rowB = W * 4u;   // bytes per packed row

    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int k = 0; k < kOthStages; ++k) mbar_init(&bar_oth[k], 1);
        for (int k = 0; k < kOwnStages; ++k) mbar_init(&bar_own[k], 1);
        mbar_fence_init();
        abort_flag = 0;
    }
    __syncthreads();

    // issue the copies of other-colour plane xp (periodic) into stage st
    auto load_oth = [&](int xp, int st) {
        const int xw = xp < 0 ? xp + nx : (xp >= nx ? xp - nx : xp);
        const uint32_t rb = ((uint32_t)xw * ny + y0) * W;            // first slab row
        const uint32_t ym = (y0 == 0 ? (uint32_t)ny - 1 : y0 - 1);
        const uint32_t yp = (y0 + RS == (uint32_t)ny ? 0u : y0 + RS);
        const uint32_t rm = ((uint32_t)xw * ny + ym) * W, rp = ((uint32_t)xw * ny + yp) * W;
        mbar_expect_tx(&bar_oth[st], 3u * (RS + 2u) * rowB);
        float* d = oth_s + st * oth_plane;
        for (int c = 0; c < 3; ++c) {
            const float* g = gs + (int64_t)c * N + oth_base;
            float* dc = d + c * (RS + 2u) * W;
            bulk_g2s(dc, g + rm, rowB, &bar_oth[st]);
            bulk_g2s(dc + W, g + rb, RS * rowB, &bar_oth[st]);
            bulk_g2s(dc + (RS + 1u) * W, g + rp, rowB, &bar_oth[st]);
        }
    };
    auto load_own = [&](int xp, int st) {
        const uint32_t rb = ((uint32_t)xp * ny + y0) * W;
        mbar_expect_tx(&bar_own[st], 3u * RS * rowB);
        float* d = own_s + st * own_plane;
        for (int c = 0; c < 3; ++c)
            bulk_g2s(d + c * RS * W, gs + (int64_t)c * N + own_base + rb, RS * rowB, &bar_own[st]);
    };

    // prologue: other planes x0-1 .. x0+2, own planes x0, x0+1
    const int nsteps = x1 - x0;
    if (tid == 0) {
        for (int k = 0; k < 4 && k - 1 < nsteps + 1; ++k) load_oth(x0 - 1 + k, k);
        for (int k = 0; k < 2 && k < nsteps; ++k) load_own(x0 + k, k);
    }
    // relative other plane k (= plane x0-1+k) is the (k / kOthStages)-th fill of stage
    // k % kOthStages, so its completion phase has parity (k / kOthStages) & 1; likewise own
    // plane k in stage k % kOwnStages.
    auto par_oth = [](int k) { return (uint32_t)((k / kOthStages) & 1); };
    auto par_own = [](int k) { return (uint32_t)((k / kOwnStages) & 1); };
    v2 de = V(0.f), dmx = V(0.f), dmy = V(0.f), dmz = V(0.f);
    const uint32_t tx = threadIdx.x % (W / 2u), r = threadIdx.x / (W / 2u);
    const bool active = r < RS;
    const uint32_t j = 2u * tx;
    const uint32_t y = y0 + r;
    int oth_issued = 4;   // other planes issued so far (relative index x0-1+k)
    int own_issued = 2;
    bool ok = true;
    int s = 0;
    for (; s < nsteps; ++s) {
        const int x = x0 + s;
        // stages of other planes x-1, x, x+1 are (s, s+1, s+2) % kOthStages
        const int so_m = s % kOthStages, so_0 = (s + 1) % kOthStages, so_p = (s + 2) % kOthStages;
        const int sw_ = s % kOwnStages;
        if (s == 0) {
            ok = ok && mbar_wait(&bar_oth[so_m], par_oth(s));
            ok = ok && mbar_wait(&bar_oth[so_0], par_oth(s + 1));
        }
        ok = ok && mbar_wait(&bar_oth[so_p], par_oth(s + 2));
        ok = ok && mbar_wait(&bar_own[sw_], par_own(s));
        if (!ok) abort_flag = 1;
        if (__syncthreads_or(!ok)) break;
        if (active) {
            const float* om = oth_s + so_m * oth_plane;   // plane x-1
            const float* o0 = oth_s + so_0 * oth_plane;   // plane x
            const float* op = oth_s + so_p * oth_plane;   // plane x+1
            const float* ow = own_s + sw_ * own_plane;
            const uint32_t RW = (RS + 2u) * W;            // floats per component, other stage
            auto l2 = [](const float* b, uint32_t o) { return *reinterpret_cast<const v2*>(b + o); };
            const uint32_t oc = (r + 1u) * W + j;       // this row inside an other stage
            v23 sv = {l2(ow, r * W + j), l2(ow, RS * W + r * W + j), l2(ow, 2u * RS * W + r * W + j)};
            const v23 px = {l2(op, oc), l2(op, RW + oc), l2(op, 2u * RW + oc)};
            const v23 mx = {l2(om, oc), l2(om, RW + oc), l2(om, 2u * RW + oc)};
            const v23 py = {l2(o0, oc + W), l2(o0, RW + oc + W), l2(o0, 2u * RW + oc + W)};
            const v23 my = {l2(o0, oc - W), l2(o0, RW + oc - W), l2(o0, 2u * RW + oc - W)};
            const v23 oz = {l2(o0, oc), l2(o0, RW + oc), l2(o0, 2u * RW + oc)};
            const uint32_t p = ((uint32_t)x + y + (uint32_t)colour) & 1u;
            const uint32_t je = p ? (j + 2 == W ? 0u : j + 2) : (j == 0 ? W - 1 : j - 1);
            const uint32_t oe = (r + 1u) * W + je;
            const float ex = o0[oe], ey = o0[RW + oe], ez = o0[2u * RW + oe];
            v23 zp, zm;
            if (p) { zp = {make_float2(oz.x.y, ex), make_float2(oz.y.y, ey), make_float2(oz.z.y, ez)}; zm = oz; }
            else { zp = oz; zm = {make_float2(ex, oz.x.x), make_float2(ey, oz.y.x), make_float2(ez, oz.z.x)}; }
            const v2 J = V(H.J);
            v23 h;
            h.x = mul(J, add(add(add(px.x, mx.x), add(py.x, my.x)), add(zp.x, zm.x)));
            h.y = mul(J, add(add(add(px.y, mx.y), add(py.y, my.y)), add(zp.y, zm.y)));
            h.z = mul(J, add(add(add(px.z, mx.z), add(py.z, my.z)), add(zp.z, zm.z)));
            if (DMI == 1) {
                const v2 D = V(H.D[1][0]);
                h.x = fma2(D, sub(sub(zm.y, zp.y), sub(my.z, py.z)), h.x);
                h.y = fma2(D, sub(sub(mx.z, px.z), sub(zm.x, zp.x)), h.y);
                h.z = fma2(D, sub(sub(my.x, py.x), sub(mx.y, px.y)), h.z);
            } else if (DMI == 2) {
                const v2 D = V(H.D[2][0]);
                h.x = fma2(D, sub(px.z, mx.z), h.x);
                h.y = fma2(D, sub(py.z, my.z), h.y);
                h.z = fma2(D, sub(sub(mx.x, px.x), sub(py.y, my.y)), h.z);
            } else if (DMI == 3) {
                const v23 nb[6] = {px, mx, py, my, zp, zm};
#pragma unroll
                for (int k = 0; k < 6; ++k) {
                    const v2 dx = V(H.D[k][0]), dy = V(H.D[k][1]), dz = V(H.D[k][2]);
                    h.x = add(h.x, sub(mul(nb[k].y, dz), mul(nb[k].z, dy)));
                    h.y = add(h.y, sub(mul(nb[k].z, dx), mul(nb[k].x, dz)));
                    h.z = add(h.z, sub(mul(nb[k].x, dy), mul(nb[k].y, dx)));
                }
            }
            h.z = sub(h.z, V(H.Bz));
            const uint32_t row = (uint32_t)x * ny + y;
            const uint32_t i0 = row * (uint32_t)a.nz + 2u * j + p;
            const uint32_t cw = (a.ensemble << 8) | kTagSweep;
            const uint4 ra = philox_rk(make_uint4(i0, sweep, rep, cw), P.rk);
            const uint4 rb = philox_rk(make_uint4(i0 + 2u, sweep, rep, cw), P.rk);
            const v23 sp = propose2<MOVE>(sv, ra, rb, a.r);
            const v23 d = {sub(sp.x, sv.x), sub(sp.y, sv.y), sub(sp.z, sv.z)};
            v2 dE = fma2(d.x, h.x, fma2(d.y, h.y, mul(d.z, h.z)));
            if (HAS_K) {
                const v2 e1 = fma2(sp.x, V(H.kx), fma2(sp.y, V(H.ky), mul(sp.z, V(H.kz))));
                const v2 e0 = fma2(sv.x, V(H.kx), fma2(sv.y, V(H.ky), mul(sv.z, V(H.kz))));
                dE = fma2(V(-H.K), mul(sub(e1, e0), add(e1, e0)), dE);
            }
            if (!(dE.x == dE.x) || !(dE.y == dE.y)) atomicOr(a.status, kStatNan);
            const v2 t = mul(V(-beta2), dE);
            const v2 u3 = u01x2(ra.w, rb.w);
            const bool acc0 = (dE.x <= 0.f) || (u3.x < ax_ex2(t.x));
            const bool acc1 = (dE.y <= 0.f) || (u3.y < ax_ex2(t.y));
            const v2 m = make_float2(acc0 ? 1.f : 0.f, acc1 ? 1.f : 0.f);
            de = fma2(m, dE, de);
            dmx = fma2(m, d.x, dmx);
            dmy = fma2(m, d.y, dmy);
            dmz = fma2(m, d.z, dmz);
            if (acc0 | acc1) {
                const uint32_t o = own_base + row * W + j;
                *reinterpret_cast<v2*>(gs + o) = make_float2(acc0 ? sp.x.x : sv.x.x, acc1 ? sp.x.y : sv.x.y);
                *reinterpret_cast<v2*>(gs + N + o) = make_float2(acc0 ? sp.y.x : sv.y.x, acc1 ? sp.y.y : sv.y.y);
                *reinterpret_cast<v2*>(gs + 2 * N + o) = make_float2(acc0 ? sp.z.x : sv.z.x, acc1 ? sp.z.y : sv.z.y);
            }
        }
        // stages of other plane x-1 and own plane x are free once every thread passed here
        __syncthreads();
        if (tid == 0) {
            // other planes needed up to x1 (relative index nsteps + 1); refill the freed stage
            if (oth_issued <= nsteps + 1) { load_oth(x0 - 1 + oth_issued, oth_issued % kOthStages); ++oth_issued; }
            if (own_issued < nsteps) { load_own(x0 + own_issued, own_issued % kOwnStages); ++own_issued; }
        }
    }
    if (abort_flag) {
        // drain: every issued copy completes before the block's shared memory is released
        if (tid == 0) {
            atomicOr(a.status, kStatTimeout);
            // planes from the failed step on may still have copies in flight
            for (int k = s; k < oth_issued; ++k) mbar_wait_drain(&bar_oth[k % kOthStages], par_oth(k));
            for (int k = s; k < own_issued; ++k) mbar_wait_drain(&bar_own[k % kOwnStages], par_own(k));
        }
        __syncthreads();
        return;
    }
    if (a.partials) {
        __shared__ float red[4][kTmaMaxThreads / 32];
        const int lane = tid & 31, w = tid >> 5;
        const int nw = (blockDim.x + 31) >> 5;
        float v0 = warp_sum(de.x + de.y), v1 = warp_sum(dmx.x + dmx.y);
        float v2_ = warp_sum(dmy.x + dmy.y), v3 = warp_sum(dmz.x + dmz.y);
        if (lane == 0) { red[0][w] = v0; red[1][w] = v1; red[2][w] = v2_; red[3][w] = v3; }
        __syncthreads();
        if (tid < 4) {
            double t = 0.0;
            for (int k = 0; k < nw; ++k) t += (double)red[tid][k];
            // one partial slot per (slab, chunk) of this replica
            const uint32_t slot = slab * P.nchunk + chunk;
            a.partials[((int64_t)rep * a.slots_per_rep + slot) * 4 + tid] += t;
        }
    }
}

// Geometry of the TMA pass for a mesh, or false if it does not apply.
static bool tma_geometry(int nx, int ny, int nz, uint32_t* RS, uint32_t* XC) {
    if (nz % 8) return false;                     // 16-byte rows and alignment
    const int pairs = nz / 4;                     // threads per packed row
    if (pairs > kTmaMaxThreads) return false;
    int best = 0;
    for (int d = 1; d <= ny; ++d)
        if (ny % d == 0 && d * pairs <= kTmaMaxThreads) best = d;
    if (best < 1) return false;
    *RS = (uint32_t)best;
    *XC = (uint32_t)std::min(nx, 16);
    return true;
}

bool cb_tma_supported(int nx, int ny, int nz) {
    uint32_t rs, xc;
    return tma_geometry(nx, ny, nz, &rs, &xc);
}

int cb_tma_slots_per_rep(int nx, int ny, int nz) {
    uint32_t rs, xc;
    if (!tma_geometry(nx, ny, nz, &rs, &xc)) return 0;
    return (int)((ny / rs) * ((nx + xc - 1) / xc));
}

template <int MOVE, int DMI>
static int tma_dispatch(const TmaParams& P, dim3 g, dim3 b, size_t sm, bool hk, cudaStream_t s) {
    auto kern = hk ? k_cb_tma<MOVE, DMI, true> : k_cb_tma<MOVE, DMI, false>;
    ISG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    kern<<<g, b, sm, s>>>(P);
    return ISING_OK;
}

int launch_cb_tma(const CbLaunch& a, int move, int dmi, cudaStream_t s) {
    const int nrep = a.seg[0].n_rep + (a.n_seg > 1 ? a.seg[1].n_rep : 0);
    if (nrep <= 0) return ISING_OK;
    TmaParams P;
    P.a = a;
    uint32_t RS, XC;
    if (!tma_geometry(a.nx, a.ny, a.nz, &RS, &XC)) return fail(ISING_ERR_ARG, "mesh shape not supported by the TMA pass");
    P.W = (uint32_t)(a.nz / 2);
    P.RS = RS;
    P.XC = XC;
    P.nslab = (uint32_t)a.ny / RS;
    P.nchunk = ((uint32_t)a.nx + XC - 1) / XC;
    P.half = (uint32_t)(a.natoms / 2);
    {
        philox_round_keys(a.seed, P.rk);
    }
    const size_t sm = sizeof(float) * ((size_t)kOthStages * 3 * (RS + 2) * P.W + (size_t)kOwnStages * 3 * RS * P.W);
    // whole warps only: the block reduction shuffles with a full mask
    const uint32_t nthr = ((RS * (P.W / 2) + 31u) / 32u) * 32u;
    dim3 g(P.nchunk * P.nslab * (uint32_t)nrep), b(nthr);
    const bool hk = a.ham.K != 0.f;
    int st = ISING_OK;
#define ISG_T(M, D) st = tma_dispatch<M, D>(P, g, b, sm, hk, s)
    if (move == 0) {
        switch (dmi) { case 0: ISG_T(0, 0); break; case 1: ISG_T(0, 1); break;
                       case 2: ISG_T(0, 2); break; default: ISG_T(0, 3); }
    } else {
        switch (dmi) { case 0: ISG_T(1, 0); break; case 1: ISG_T(1, 1); break;
                       case 2: ISG_T(1, 2); break; default: ISG_T(1, 3); }
    }
#undef ISG_T
    if (st != ISING_OK) return st;
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}

}  // namespace isg
