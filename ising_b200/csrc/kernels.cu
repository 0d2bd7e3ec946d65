// kernels.cu -- sm_100a kernels of libisinggpu (grid-launched forms).
//
// Layout in HBM: per replica three FP32 planes (Sx[N], Sy[N], Sz[N]) in the reference's atom
// order (z fastest for one atom per cell); replicas follow each other.  FP64 is used only in
// per-replica accumulators and in the parity reductions.
#include <cstdio>

#include "internal.h"
#include "exchange.cuh"
#include "winding.cuh"

namespace isg {

// ================================================================= helpers
template <typename T>
__device__ __forceinline__ void block_sum4(T v0, T v1, T v2, T v3, T* out /* smem 4 */) {
    __shared__ T red[4][32];
    v0 = warp_sum(v0); v1 = warp_sum(v1); v2 = warp_sum(v2); v3 = warp_sum(v3);
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int lane = tid & 31, wid = tid >> 5;
    const int nw = (blockDim.x * blockDim.y + 31) >> 5;
    if (lane == 0) { red[0][wid] = v0; red[1][wid] = v1; red[2][wid] = v2; red[3][wid] = v3; }
    __syncthreads();
    if (wid == 0) {
        T a = lane < nw ? red[0][lane] : T(0), b = lane < nw ? red[1][lane] : T(0);
        T c = lane < nw ? red[2][lane] : T(0), d = lane < nw ? red[3][lane] : T(0);
        a = warp_sum(a); b = warp_sum(b); c = warp_sum(c); d = warp_sum(d);
        if (lane == 0) { out[0] = a; out[1] = b; out[2] = c; out[3] = d; }
    }
}

// ================================================================= general crystal sweep
// One colour class of a greedy colouring over an arbitrary unit cell: the site list of the
// class is read, each site's neighbours come from its sublattice stencil (cell offset plus
// sublattice) held in shared memory.
constexpr int kGenThreads = 256;
constexpr int kGenSitesPerThread = 4;

int general_slots_for(int n_sites) {
    int per = kGenThreads * kGenSitesPerThread;
    return (n_sites + per - 1) / per;
}

__device__ __forceinline__ void decode_atom(int64_t at, int nsub, int ny, int nz, int* ix, int* iy,
                                            int* iz, int* sub) {
    *sub = (int)(at % nsub);
    const int64_t cell = at / nsub;
    *iz = (int)(cell % nz);
    const int64_t r = cell / nz;
    *iy = (int)(r % ny);
    *ix = (int)(r / ny);
}

// local field of atom (ix,iy,iz,sub) from its stencil in shared memory
__device__ __forceinline__ f3 stencil_field(const float* sx, const float* sy, const float* sz,
                                            const Slot* sl, int cnt, int ix, int iy, int iz,
                                            const Layout& L) {
    f3 h = {0.f, 0.f, 0.f};
    for (int q = 0; q < cnt; ++q) {
        const Slot e = sl[q];
        const int jx = wrap_any(ix + e.dx, L.nx), jy = wrap_any(iy + e.dy, L.ny), jz = wrap_any(iz + e.dz, L.nz);
        const int64_t j = sidx(L, jx, jy, jz, e.sub);
        const f3 sj = {sx[j], sy[j], sz[j]};
        const f3 c = cross(sj, mk(e.Dx, e.Dy, e.Dz));
        h.x += fmaf(e.w, sj.x, c.x);
        h.y += fmaf(e.w, sj.y, c.y);
        h.z += fmaf(e.w, sj.z, c.z);
    }
    return h;
}

// Metropolis update of one site (ix, iy, iz, sub), reference atom index `at`, with the local
// field of its stencil; accepted moves add to the running sums.  RK: Philox with the launch's
// precomputed round keys (constant-bank operands; BCC 96^3 x 16 5.56e10 -> 6.44e10
// updates/s); false: the key schedule computed in registers, for loops that run several
// updates per thread, where the compiler keeps the 20 round keys in registers instead
// (hyper-kagome's 4 pairs per thread: 6.12e10 -> 5.07e10 with round keys at 48 registers).
// Both give the same numbers.
template <int MOVE, bool RK = true>
__device__ __forceinline__ void site_update(const GeneralLaunch& a, f3 h, int64_t si, int64_t at, float* sx,
                                            float* sy, float* sz, uint32_t sweep, int rep, float beta, float& de,
                                            float& dmx, float& dmy, float& dmz) {
    const HamDev& H = a.ham;
    h.z -= H.Bz;
    if (a.demag) {   // -mu_0 S.H of calculateHeisenbergEnergy (src/energyMin.f90:163-167)
        const int64_t N = a.natoms;
        h.x = fmaf(-a.mu0, a.demag[si], h.x);
        h.y = fmaf(-a.mu0, a.demag[N + si], h.y);
        h.z = fmaf(-a.mu0, a.demag[2 * N + si], h.z);
    }
    const f3 s = {sx[si], sy[si], sz[si]};
    const uint4 c4 = make_uint4((uint32_t)at, sweep, (uint32_t)rep, (a.ensemble << 8) | kTagSweep);
    const uint4 r4 = RK ? philox_rk(c4, a.rk) : philox4x32<10>(c4, philox_key(a.seed));
    const f3 sp = propose<MOVE>(s, u01(r4.x), u01(r4.y), u01(r4.z), a.r);
    // every operation rounded as written, so that a lane of site_update_pair gives the same
    const float dx = __fsub_rn(sp.x, s.x), dy = __fsub_rn(sp.y, s.y), dz = __fsub_rn(sp.z, s.z);
    float dE = fmaf(dx, h.x, fmaf(dy, h.y, __fmul_rn(dz, h.z)));
    if (H.K != 0.f) {
        const float e1 = fmaf(sp.x, H.kx, fmaf(sp.y, H.ky, __fmul_rn(sp.z, H.kz)));
        const float e0 = fmaf(s.x, H.kx, fmaf(s.y, H.ky, __fmul_rn(s.z, H.kz)));
        dE = fmaf(-H.K, __fmul_rn(__fsub_rn(e1, e0), __fadd_rn(e1, e0)), dE);
    }
    if (!(dE == dE)) atomicOr(a.status, kStatNan);
    if ((dE <= 0.f) || (u01(r4.w) < __expf(-beta * dE))) {
        sx[si] = sp.x; sy[si] = sp.y; sz[si] = sp.z;
        de += dE; dmx += dx; dmy += dy; dmz += dz;
    }
}

// The update of the site pair (si, si + 1) of one row (si even; reference atoms at0, at1)
// with its two fields in the lanes of packed FP32x2 (hx, hy, hz): the pair's spins are read as
// one aligned pair per component, the proposals (propose2), energy changes and anisotropy run
// in packed arithmetic, the decisions per lane.  Each lane performs site_update's operations
// in the same order and rounding, so the pair equals two site_update calls bit for bit.
template <int MOVE, bool RK = true>
__device__ __forceinline__ void site_update_pair(const GeneralLaunch& a, float2 hx, float2 hy, float2 hz, int64_t si,
                                                 uint32_t at0, uint32_t at1, float* sx, float* sy, float* sz,
                                                 uint32_t sweep, int rep, float beta, float& de, float& dmx, float& dmy,
                                                 float& dmz) {
    const HamDev& H = a.ham;
    hz = __fadd2_rn(hz, make_float2(-H.Bz, -H.Bz));
    if (a.demag) {   // -mu_0 S.H of calculateHeisenbergEnergy (src/energyMin.f90:163-167)
        const int64_t N = a.natoms;
        const float2 nm = make_float2(-a.mu0, -a.mu0);
        hx = __ffma2_rn(nm, *reinterpret_cast<const float2*>(a.demag + si), hx);
        hy = __ffma2_rn(nm, *reinterpret_cast<const float2*>(a.demag + N + si), hy);
        hz = __ffma2_rn(nm, *reinterpret_cast<const float2*>(a.demag + 2 * N + si), hz);
    }
    float2 s[3] = {*reinterpret_cast<const float2*>(sx + si), *reinterpret_cast<const float2*>(sy + si),
                   *reinterpret_cast<const float2*>(sz + si)};
    const uint32_t cw = (a.ensemble << 8) | kTagSweep;
    const uint4 ca = make_uint4(at0, sweep, (uint32_t)rep, cw), cb = make_uint4(at1, sweep, (uint32_t)rep, cw);
    const uint4 ra = RK ? philox_rk(ca, a.rk) : philox4x32<10>(ca, philox_key(a.seed));
    const uint4 rb = RK ? philox_rk(cb, a.rk) : philox4x32<10>(cb, philox_key(a.seed));
    float2 sp[3];
    propose2<MOVE>(s, ra, rb, a.r, sp);
    const float2 m1 = make_float2(-1.f, -1.f);
    const float2 dx = __ffma2_rn(s[0], m1, sp[0]), dy = __ffma2_rn(s[1], m1, sp[1]), dz = __ffma2_rn(s[2], m1, sp[2]);
    float2 dE = __ffma2_rn(dx, hx, __ffma2_rn(dy, hy, __fmul2_rn(dz, hz)));
    if (H.K != 0.f) {
        const float2 kx = make_float2(H.kx, H.kx), ky = make_float2(H.ky, H.ky), kz = make_float2(H.kz, H.kz);
        const float2 e1 = __ffma2_rn(sp[0], kx, __ffma2_rn(sp[1], ky, __fmul2_rn(sp[2], kz)));
        const float2 e0 = __ffma2_rn(s[0], kx, __ffma2_rn(s[1], ky, __fmul2_rn(s[2], kz)));
        dE = __ffma2_rn(make_float2(-H.K, -H.K), __fmul2_rn(__ffma2_rn(e0, m1, e1), __fadd2_rn(e1, e0)), dE);
    }
    if (!(dE.x == dE.x) || !(dE.y == dE.y)) atomicOr(a.status, kStatNan);
    const bool acc0 = (dE.x <= 0.f) || (u01(ra.w) < __expf(-beta * dE.x));
    const bool acc1 = (dE.y <= 0.f) || (u01(rb.w) < __expf(-beta * dE.y));
    if (acc0 && acc1) {
        *reinterpret_cast<float2*>(sx + si) = sp[0];
        *reinterpret_cast<float2*>(sy + si) = sp[1];
        *reinterpret_cast<float2*>(sz + si) = sp[2];
    } else if (acc0) {
        sx[si] = sp[0].x; sy[si] = sp[1].x; sz[si] = sp[2].x;
    } else if (acc1) {
        sx[si + 1] = sp[0].y; sy[si + 1] = sp[1].y; sz[si + 1] = sp[2].y;
    }
    if (acc0) { de += dE.x; dmx += dx.x; dmy += dy.x; dmz += dz.x; }
    if (acc1) { de += dE.y; dmx += dx.y; dmy += dy.y; dmz += dz.y; }
}

template <int MOVE>
__device__ __forceinline__ void general_site(const GeneralLaunch& a, const Slot* sl, const int* cnt, float* sx,
                                             float* sy, float* sz, int64_t at, int ix, int iy, int iz, int sub,
                                             uint32_t sweep, int rep, float beta, float& de, float& dmx, float& dmy,
                                             float& dmz) {
    const f3 h = stencil_field(sx, sy, sz, sl + sub * kMaxSlots, cnt[sub], ix, iy, iz, a.layout);
    site_update<MOVE>(a, h, sidx(a.layout, ix, iy, iz, sub), at, sx, sy, sz, sweep, rep, beta, de, dmx, dmy, dmz);
}

template <int MOVE>
__global__ void __launch_bounds__(kGenThreads) k_general_colour(GeneralLaunch a) {
    extern __shared__ unsigned char smem_raw[];
    Slot* sl = reinterpret_cast<Slot*>(smem_raw);
    int* cnt = reinterpret_cast<int*>(sl + a.st.nsub * kMaxSlots);
    for (int q = threadIdx.x; q < a.st.nsub * kMaxSlots; q += blockDim.x) sl[q] = a.st.slots[q];
    for (int q = threadIdx.x; q < a.st.nsub; q += blockDim.x) cnt[q] = a.st.count[q];
    __syncthreads();
    const int rl = blockIdx.y;
    const int rep = a.rep_first + rl;
    const int64_t N = a.natoms;
    float* __restrict__ sx = a.spins + (int64_t)rl * 3 * N;
    float* __restrict__ sy = sx + N;
    float* __restrict__ sz = sy + N;
    const uint32_t sweep = a.sweep_ctr[rep] + a.sweep_offset;
    const float beta = (float)a.beta_rep[rep];
    float de = 0.f, dmx = 0.f, dmy = 0.f, dmz = 0.f;
    const int base = blockIdx.x * blockDim.x * kGenSitesPerThread;
    for (int it = 0; it < kGenSitesPerThread; ++it) {
        const int t = base + it * blockDim.x + threadIdx.x;
        if (t >= a.n_sites) break;
        const int64_t at = a.sites[t];
        int ix, iy, iz, sub;
        decode_atom(at, a.nsub, a.ny, a.nz, &ix, &iy, &iz, &sub);
        general_site<MOVE>(a, sl, cnt, sx, sy, sz, at, ix, iy, iz, sub, sweep, rep, beta, de, dmx, dmy, dmz);
    }
    if (a.partials) {
        __shared__ double tot[4];
        block_sum4<double>(de, dmx, dmy, dmz, tot);
        if (threadIdx.x == 0) {
            double* p = a.partials + ((int64_t)rep * a.slots_per_rep + a.slot_base + blockIdx.x) * 4;
            p[0] += tot[0]; p[1] += tot[1]; p[2] += tot[2]; p[3] += tot[3];
        }
    }
}

// One class of the octant colouring: thread t of the class updates the site of storage rank
// rank0 + t / q8 at packed cell t % q8 of the octant, so the own reads and writes of a warp
// are consecutive and so are its reads through each stencil slot (the packed cells of a
// neighbour octant move in step).  Same arithmetic and Philox keys as k_general_colour.
template <int MOVE>
__global__ void __launch_bounds__(kGenThreads) k_octant_colour(GeneralLaunch a, int oct, int rank0, int nrank) {
    extern __shared__ unsigned char smem_raw[];
    Slot* sl = reinterpret_cast<Slot*>(smem_raw);
    int* cnt = reinterpret_cast<int*>(sl + a.st.nsub * kMaxSlots);
    for (int q = threadIdx.x; q < a.st.nsub * kMaxSlots; q += blockDim.x) sl[q] = a.st.slots[q];
    for (int q = threadIdx.x; q < a.st.nsub; q += blockDim.x) cnt[q] = a.st.count[q];
    __syncthreads();
    const int rl = blockIdx.y;
    const int rep = a.rep_first + rl;
    const int64_t N = a.natoms;
    float* __restrict__ sx = a.spins + (int64_t)rl * 3 * N;
    float* __restrict__ sy = sx + N;
    float* __restrict__ sz = sy + N;
    const uint32_t sweep = a.sweep_ctr[rep] + a.sweep_offset;
    const float beta = (float)a.beta_rep[rep];
    const Layout& L = a.layout;
    const int64_t q8 = L.q8, n = q8 * nrank;
    const int hy = a.ny >> 1, hz = a.nz >> 1;
    const int ox = (oct >> 2) & 1, oy = (oct >> 1) & 1, oz = oct & 1;
    float de = 0.f, dmx = 0.f, dmy = 0.f, dmz = 0.f;
    const int64_t base = (int64_t)blockIdx.x * blockDim.x * kGenSitesPerThread;
    for (int it = 0; it < kGenSitesPerThread; ++it) {
        const int64_t t = base + it * blockDim.x + threadIdx.x;
        if (t >= n) break;
        const int rk = rank0 + (int)(t / q8);
        const int64_t pc = t - (int64_t)(rk - rank0) * q8;
        const int Z = (int)(pc % hz);
        const int64_t r = pc / hz;
        const int Y = (int)(r % hy), X = (int)(r / hy);
        const int ix = 2 * X + ox, iy = 2 * Y + oy, iz = 2 * Z + oz, sub = L.sofr[rk];
        const int64_t at = (((int64_t)ix * a.ny + iy) * a.nz + iz) * a.nsub + sub;
        general_site<MOVE>(a, sl, cnt, sx, sy, sz, at, ix, iy, iz, sub, sweep, rep, beta, de, dmx, dmy, dmz);
    }
    if (a.partials) {
        __shared__ double tot[4];
        block_sum4<double>(de, dmx, dmy, dmz, tot);
        if (threadIdx.x == 0) {
            double* p = a.partials + ((int64_t)rep * a.slots_per_rep + a.slot_base + blockIdx.x) * 4;
            p[0] += tot[0]; p[1] += tot[1]; p[2] += tot[2]; p[3] += tot[3];
        }
    }
}

// The same class with the stencil resolved per class: a neighbour of the site at packed cell
// (X, Y, Z) of octant o through cell offset d lies in octant (o + d) & 1 per axis, at packed
// cell X + floor((o_x + d_x) / 2) (and so on) of its sublattice's plane, so per (rank, slot)
// the plane base and three packed offsets are fixed for the whole class.  The block resolves
// them into shared memory once; a site then needs three compare-and-wrap steps and one
// multiply-add chain per neighbour instead of the cell-coordinate modulo and octant decode
// of sidx.  Every packed offset is within one period (the launcher checks), the summation
// order is the stencil's, and the update is the one of k_octant_colour, bit for bit.
struct __align__(16) OctSlot {
    int plane;               // (octant * nsub + storage rank) * q8 of the neighbour
    int8_t ex, ey, ez, pad;  // packed-cell offsets
    float w, Dx, Dy, Dz;
    float pad2[2];           // 32 bytes: two 16-byte shared-memory loads
};
struct OctDims {
    FastDiv q8, hz, hy, hyz;
    int hx, hyi, hzi;
    FastDiv q8h;             // by q8 / 2 (site pairs of k_octant_pair)
};

// Per launch the block stencils of a list of octant blocks (octant << 4 | storage rank):
// table entry b * mc + slot, and per block its sublattice, slot count, octant and storage base.
// The kernels take the launch structs as __grid_constant__ parameters, so the block list and
// the layout tables are indexed in the parameter space (no per-thread copy).
struct OctBlockSmem {
    OctSlot* tab;
    int *sub, *cnt, *oct;
    uint32_t* base;
};
__device__ __forceinline__ OctBlockSmem octant_smem(unsigned char* raw, int nb, int mc) {
    OctBlockSmem m;
    m.tab = reinterpret_cast<OctSlot*>(raw);
    m.sub = reinterpret_cast<int*>(m.tab + nb * mc);
    m.cnt = m.sub + nb;
    m.oct = m.cnt + nb;
    m.base = reinterpret_cast<uint32_t*>(m.oct + nb);
    return m;
}
size_t octant_smem_bytes(int nb, int mc) { return (size_t)nb * mc * sizeof(OctSlot) + 4 * (size_t)nb * sizeof(int); }

__device__ __forceinline__ void octant_table(const GeneralLaunch& a, const OctBlockSmem& m, int mc, const uint8_t* code,
                                             int nb) {
    const int q8 = (int)a.layout.q8;
    for (int e = threadIdx.x; e < nb * mc; e += blockDim.x) {
        const int b = e / mc, q = e - b * mc;
        const int oct = code[b] >> 4;
        const int ox = (oct >> 2) & 1, oy = (oct >> 1) & 1, oz = oct & 1;
        const int sub = a.layout.sofr[code[b] & 15];
        OctSlot o{};
        if (q < a.st.count[sub]) {
            const Slot sl = a.st.slots[sub * kMaxSlots + q];
            const int tx = ox + sl.dx, ty = oy + sl.dy, tz = oz + sl.dz;
            const int o2 = ((tx & 1) << 2) | ((ty & 1) << 1) | (tz & 1);
            o.plane = (o2 * a.nsub + a.layout.srank[sl.sub]) * q8;
            o.ex = (int8_t)(tx >> 1); o.ey = (int8_t)(ty >> 1); o.ez = (int8_t)(tz >> 1);
            o.w = sl.w; o.Dx = sl.Dx; o.Dy = sl.Dy; o.Dz = sl.Dz;
        }
        m.tab[e] = o;
    }
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        const int oct = code[b] >> 4, rank = code[b] & 15;
        m.sub[b] = a.layout.sofr[rank];
        m.cnt[b] = a.st.count[m.sub[b]];
        m.oct[b] = oct;
        m.base[b] = (uint32_t)((oct * a.nsub + rank) * q8);
    }
}

// One bond's term of a site's local field, h += w S_j + S_j x D, every operation rounded as
// written; k_octant_pair computes the same terms for its two sites in the lanes of FP32x2, so
// the octant kernels agree bit for bit.
__device__ __forceinline__ void bond_term(f3& h, const f3& sj, const OctSlot& o) {
    const float cx = fmaf(sj.y, o.Dz, __fmul_rn(sj.z, -o.Dy));
    const float cy = fmaf(sj.z, o.Dx, __fmul_rn(sj.x, -o.Dz));
    const float cz = fmaf(sj.x, o.Dy, __fmul_rn(sj.y, -o.Dx));
    h.x = __fadd_rn(h.x, fmaf(o.w, sj.x, cx));
    h.y = __fadd_rn(h.y, fmaf(o.w, sj.y, cy));
    h.z = __fadd_rn(h.z, fmaf(o.w, sj.z, cz));
}

// block sums of the four running partials: FP32 within a warp (a warp's few sites), FP64
// across warps
__device__ __forceinline__ void block_sum4_fd(float v0, float v1, float v2, float v3, double* out /* smem 4 */) {
    __shared__ double red[4][32];
    v0 = warp_sum(v0); v1 = warp_sum(v1); v2 = warp_sum(v2); v3 = warp_sum(v3);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane == 0) { red[0][wid] = v0; red[1][wid] = v1; red[2][wid] = v2; red[3][wid] = v3; }
    __syncthreads();
    if (threadIdx.x < 4) {
        double t = 0.0;
        for (int k = 0; k < nw; ++k) t += red[threadIdx.x][k];
        out[threadIdx.x] = t;
    }
    __syncthreads();
}

// A class given as a list of octant blocks (the blocks of one class share no bond, so they
// are updated at once): thread t takes site t % q8 of block t / q8, SPT sites per thread
// (consecutive runs of blockDim.x sites), so that the block's set-up and its reduction are
// shared by SPT x 256 sites where a launch has enough of them
template <int MOVE, int SPT>
__global__ void __launch_bounds__(kGenThreads) k_octant_fast(const __grid_constant__ GeneralLaunch a, OctDims od,
                                                              const __grid_constant__ OctBlocks bl) {
    extern __shared__ __align__(16) unsigned char oct_smem[];
    const int mc = a.oct_maxcnt, nb = bl.n;
    const OctBlockSmem m = octant_smem(oct_smem, nb, mc);
    octant_table(a, m, mc, bl.code, nb);
    __syncthreads();
    const int rl = blockIdx.y;
    const int rep = a.rep_first + rl;
    const int64_t N = a.natoms;
    float* __restrict__ sx = a.spins + (int64_t)rl * 3 * N;
    float* __restrict__ sy = sx + N;
    float* __restrict__ sz = sy + N;
    const uint32_t sweep = a.sweep_ctr[rep] + a.sweep_offset;
    const float beta = (float)a.beta_rep[rep];
    const int q8 = (int)a.layout.q8;
    const uint32_t ntot = (uint32_t)q8 * (uint32_t)nb;
    const int hx = od.hx, hy = od.hyi, hz = od.hzi;
    float de = 0.f, dmx = 0.f, dmy = 0.f, dmz = 0.f;
#pragma unroll 1
    for (int it = 0; it < SPT; ++it) {
        const uint32_t t = (blockIdx.x * SPT + it) * blockDim.x + threadIdx.x;
        if (t >= ntot) break;
        const uint32_t b = fdiv(t, od.q8);
        const uint32_t pc = t - b * (uint32_t)q8;
        const uint32_t r = fdiv(pc, od.hz);
        const int Z = (int)(pc - r * (uint32_t)hz);
        const uint32_t Xu = fdiv(r, od.hy);
        const int Y = (int)(r - Xu * (uint32_t)hy), X = (int)Xu;
        const int oct = m.oct[b], sub = m.sub[b];
        const int ix = 2 * X + ((oct >> 2) & 1), iy = 2 * Y + ((oct >> 1) & 1), iz = 2 * Z + (oct & 1);
        const uint32_t at = ((uint32_t)(ix * a.ny + iy) * (uint32_t)a.nz + (uint32_t)iz) * (uint32_t)a.nsub + sub;
        const OctSlot* ts = m.tab + b * mc;
        f3 h = {0.f, 0.f, 0.f};
        const int cn = m.cnt[b];
        for (int q = 0; q < cn; ++q) {
            const OctSlot o = ts[q];
            int jx = X + o.ex, jy = Y + o.ey, jz = Z + o.ez;
            jx += jx < 0 ? hx : 0; jx -= jx >= hx ? hx : 0;
            jy += jy < 0 ? hy : 0; jy -= jy >= hy ? hy : 0;
            jz += jz < 0 ? hz : 0; jz -= jz >= hz ? hz : 0;
            const uint32_t j = (uint32_t)o.plane + (uint32_t)((jx * hy + jy) * hz + jz);
            const f3 sj = {sx[j], sy[j], sz[j]};
            bond_term(h, sj, o);
        }
        site_update<MOVE>(a, h, (int64_t)(m.base[b] + pc), (int64_t)at, sx, sy, sz, sweep, rep, beta, de, dmx, dmy,
                          dmz);
    }
    if (a.partials) {
        __shared__ double tot[4];
        block_sum4_fd(de, dmx, dmy, dmz, tot);
        if (threadIdx.x == 0) {
            double* p = a.partials + ((int64_t)rep * a.slots_per_rep + a.slot_base + blockIdx.x) * 4;
            p[0] += tot[0]; p[1] += tot[1]; p[2] += tot[2]; p[3] += tot[3];
        }
    }
}

// The same class, one pair of sites per thread: packed cells Z0 and Z0 + 1 (Z0 even, nz % 4 ==
// 0, so a pair never straddles a row) of one row.  The pair shares the row decode and, per
// stencil slot, the x/y wrap and the row base; a slot with no packed z offset reads both
// neighbours as one aligned pair per component.  Each site's field is summed in slot order
// with bond_term's operations in FP32x2 lanes, so the update equals k_octant_fast's bit for bit.
template <int MOVE, int PPT>
__global__ void __launch_bounds__(kGenThreads, 5) k_octant_pair(const __grid_constant__ GeneralLaunch a, OctDims od,
                                                                 const __grid_constant__ OctBlocks bl) {
    extern __shared__ __align__(16) unsigned char oct_smem[];
    const int mc = a.oct_maxcnt, nb = bl.n;
    const OctBlockSmem m = octant_smem(oct_smem, nb, mc);
    octant_table(a, m, mc, bl.code, nb);
    __syncthreads();
    const int rl = blockIdx.y;
    const int rep = a.rep_first + rl;
    const int64_t N = a.natoms;
    float* __restrict__ sx = a.spins + (int64_t)rl * 3 * N;
    float* __restrict__ sy = sx + N;
    float* __restrict__ sz = sy + N;
    const uint32_t sweep = a.sweep_ctr[rep] + a.sweep_offset;
    const float beta = (float)a.beta_rep[rep];
    const int hx = od.hx, hy = od.hyi, hz = od.hzi;
    const uint32_t half8 = (uint32_t)a.layout.q8 >> 1;
    const uint32_t npair = half8 * (uint32_t)nb;
    float de = 0.f, dmx = 0.f, dmy = 0.f, dmz = 0.f;
#pragma unroll 1
    for (int it = 0; it < PPT; ++it) {
        const uint32_t tp = (blockIdx.x * PPT + it) * blockDim.x + threadIdx.x;
        if (tp >= npair) break;
        const uint32_t b = fdiv(tp, od.q8h);
        const uint32_t pc0 = 2u * (tp - b * half8);
        const uint32_t r = fdiv(pc0, od.hz);
        const int Z0 = (int)(pc0 - r * (uint32_t)hz);
        const uint32_t Xu = fdiv(r, od.hy);
        const int Y = (int)(r - Xu * (uint32_t)hy), X = (int)Xu;
        const int oct = m.oct[b], sub = m.sub[b];
        const int ix = 2 * X + ((oct >> 2) & 1), iy = 2 * Y + ((oct >> 1) & 1), iz = 2 * Z0 + (oct & 1);
        const uint32_t at0 = ((uint32_t)(ix * a.ny + iy) * (uint32_t)a.nz + (uint32_t)iz) * (uint32_t)a.nsub + sub;
        const uint32_t at1 = at0 + 2u * (uint32_t)a.nsub;   // cell z + 2
        const OctSlot* ts = m.tab + b * mc;
        float2 hx2 = make_float2(0.f, 0.f), hy2 = hx2, hz2 = hx2;   // the two sites' fields
        const int cn = m.cnt[b];
        for (int q = 0; q < cn; ++q) {
            const OctSlot o = ts[q];
            int jx = X + o.ex, jy = Y + o.ey;
            jx += jx < 0 ? hx : 0; jx -= jx >= hx ? hx : 0;
            jy += jy < 0 ? hy : 0; jy -= jy >= hy ? hy : 0;
            const uint32_t rb = (uint32_t)o.plane + (uint32_t)((jx * hy + jy) * hz);
            f3 s0, s1;
            if (o.ez == 0) {   // both neighbours at Z0, Z0 + 1: one aligned pair per component
                const float2 px = *reinterpret_cast<const float2*>(sx + rb + Z0);
                const float2 py = *reinterpret_cast<const float2*>(sy + rb + Z0);
                const float2 pz = *reinterpret_cast<const float2*>(sz + rb + Z0);
                s0 = {px.x, py.x, pz.x};
                s1 = {px.y, py.y, pz.y};
            } else {
                int jz0 = Z0 + o.ez, jz1 = Z0 + 1 + o.ez;
                jz0 += jz0 < 0 ? hz : 0; jz0 -= jz0 >= hz ? hz : 0;
                jz1 += jz1 < 0 ? hz : 0; jz1 -= jz1 >= hz ? hz : 0;
                s0 = {sx[rb + jz0], sy[rb + jz0], sz[rb + jz0]};
                s1 = {sx[rb + jz1], sy[rb + jz1], sz[rb + jz1]};
            }
            // bond_term for both sites in the lanes of FP32x2
            const float2 PX = make_float2(s0.x, s1.x), PY = make_float2(s0.y, s1.y), PZ = make_float2(s0.z, s1.z);
            const float2 w2 = make_float2(o.w, o.w);
            const float2 cx = __ffma2_rn(PY, make_float2(o.Dz, o.Dz), __fmul2_rn(PZ, make_float2(-o.Dy, -o.Dy)));
            const float2 cy = __ffma2_rn(PZ, make_float2(o.Dx, o.Dx), __fmul2_rn(PX, make_float2(-o.Dz, -o.Dz)));
            const float2 cz = __ffma2_rn(PX, make_float2(o.Dy, o.Dy), __fmul2_rn(PY, make_float2(-o.Dx, -o.Dx)));
            hx2 = __fadd2_rn(hx2, __ffma2_rn(w2, PX, cx));
            hy2 = __fadd2_rn(hy2, __ffma2_rn(w2, PY, cy));
            hz2 = __fadd2_rn(hz2, __ffma2_rn(w2, PZ, cz));
        }
        const uint32_t si0 = m.base[b] + pc0;
        site_update_pair<MOVE, PPT == 1>(a, hx2, hy2, hz2, (int64_t)si0, at0, at1, sx, sy, sz, sweep, rep, beta, de, dmx,
                                         dmy, dmz);
    }
    if (a.partials) {
        __shared__ double tot[4];
        block_sum4_fd(de, dmx, dmy, dmz, tot);
        if (threadIdx.x == 0) {
            double* p = a.partials + ((int64_t)rep * a.slots_per_rep + a.slot_base + blockIdx.x) * 4;
            p[0] += tot[0]; p[1] += tot[1]; p[2] += tot[2]; p[3] += tot[3];
        }
    }
}

// ---- persistent octant engine ----------------------------------------------------------
// All sweeps of a PT round over the octant classes in ONE launch.  A task is (phase, replica,
// packed x-plane u), phase = sweep * classes + class; tasks are taken from an atomic queue in
// phase-major order, so every task a block waits for sits earlier in the queue and is held by a
// running block (no co-residency is assumed).  A task of phase p on plane u waits until the
// planes u - reach .. u + reach of its replica have finished phase p - 1: its neighbours lie
// in those planes, and the previous phase's readers of plane u lie there too.  It then
// updates every site of the class in plane u (all Y, Z, every rank of the class) exactly as
// k_octant_fast does, adds its block sums to the (replica, plane) partial slot and releases
// the plane's counter.  Ordering: thread 0 acquires the counters (ld.acquire.gpu), every
// thread acquires them again before its loads (so its SM's L1 holds no stale line), and the
// release follows __syncthreads + __threadfence.  Every wait is bounded (%globaltimer and a
// poll count); one that gives up sets kStatTimeout and raises the abort word, which stops
// every block at its next task.
__device__ __forceinline__ uint32_t oe_ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void oe_st_release(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t oe_now() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// thread 0: wait until *p >= target; false when aborted or past the bound (then aborts)
__device__ __forceinline__ bool oe_wait_ge(const OctEngineLaunch& e, int* status, const uint32_t* p, uint32_t target) {
    if (oe_ld_acquire(p) >= target) return true;
    const uint64_t t0 = oe_now();
    const uint64_t max_polls = e.wait_ns / 32u + 1024u;
    uint32_t ns = 32;
    for (uint64_t it = 0; it < max_polls; ++it) {
        __nanosleep(ns);
        if (ns < 512) ns <<= 1;
        if (oe_ld_acquire(p) >= target) return true;
        if (*(volatile const uint32_t*)e.abort) return false;
        if (oe_now() - t0 > e.wait_ns) break;
    }
    atomicOr(status, kStatTimeout);
    atomicExch(e.abort, 1u);
    __threadfence();
    return false;
}

template <int MOVE>
__global__ void __launch_bounds__(kGenThreads, 4) k_octant_engine(const __grid_constant__ GeneralLaunch a, OctDims od,
                                                                    const __grid_constant__ OctEngineLaunch e) {
    extern __shared__ __align__(16) unsigned char oe_smem[];
    const int mc = a.oct_maxcnt;
    const OctBlockSmem m = octant_smem(oe_smem, e.maxnb, mc);   // the current class's blocks
    __shared__ uint32_t s_task[3];
    __shared__ int s_go;
    __shared__ double tot[4];
    const int hx = od.hx, hy = od.hyi, hz = od.hzi;
    const uint32_t hyz = (uint32_t)hy * (uint32_t)hz;
    const int ncls = e.ncls;
    const uint32_t per_phase = (uint32_t)a.n_rep * (uint32_t)hx;
    const uint32_t total = per_phase * (uint32_t)ncls * (uint32_t)e.n_sweeps;
    const int64_t N = a.natoms;
    int cached = -1;
    uint32_t next = 0;
    if (threadIdx.x == 0) next = atomicAdd(e.head, 1u);
    for (;;) {
        if (threadIdx.x == 0) {
            int go = 0;
            const uint32_t id = next;
            if (id < total && !*(volatile const uint32_t*)e.abort) {
                const uint32_t ph = id / per_phase, rem = id - ph * per_phase;
                const uint32_t r = rem / (uint32_t)hx, u = rem - r * (uint32_t)hx;
                go = 1;
                if (ph > 0) {
                    const uint32_t* d = e.done + r * (uint32_t)hx;
                    const uint32_t target = (e.stall && ph == 1u) ? 0x40000000u : ph;
                    for (int k = -e.reach; k <= e.reach && go; ++k) {
                        int uu = ((int)u + k) % hx;
                        uu += uu < 0 ? hx : 0;
                        go = oe_wait_ge(e, a.status, d + uu, target);
                    }
                }
                s_task[0] = ph; s_task[1] = r; s_task[2] = u;
            }
            s_go = go;
        }
        __syncthreads();
        if (!s_go) break;
        if (threadIdx.x == 0) next = atomicAdd(e.head, 1u);   // prefetch; used next iteration
        const uint32_t ph = s_task[0], r = s_task[1], u = s_task[2];
        if (threadIdx.x != 0 && ph > 0) {
            const uint32_t* d = e.done + r * (uint32_t)hx;
            for (int k = -e.reach; k <= e.reach; ++k) {
                int uu = ((int)u + k) % hx;
                uu += uu < 0 ? hx : 0;
                oe_ld_acquire(d + uu);
            }
        }
        const int sw = (int)(ph / (uint32_t)ncls), c = (int)ph - sw * ncls;
        const int nb = e.start[c + 1] - e.start[c];
        if (c != cached) {   // the class's stencil, resolved as in k_octant_fast
            octant_table(a, m, mc, e.code + e.start[c], nb);
            cached = c;
            __syncthreads();
        }
        const int rep = a.rep_first + (int)r;
        float* __restrict__ sx = a.spins + (int64_t)r * 3 * N;
        float* __restrict__ sy = sx + N;
        float* __restrict__ sz = sy + N;
        const uint32_t sweep = a.sweep_ctr[rep] + a.sweep_offset + (uint32_t)sw;
        const float beta = (float)a.beta_rep[rep];
        const uint32_t nsite = (uint32_t)nb * hyz;
        const int X = (int)u;
        float de = 0.f, dmx = 0.f, dmy = 0.f, dmz = 0.f;
        for (uint32_t t = threadIdx.x; t < nsite; t += blockDim.x) {
            const uint32_t b = fdiv(t, od.hyz);
            const uint32_t rem = t - b * hyz;
            const uint32_t Yu = fdiv(rem, od.hz);
            const int Z = (int)(rem - Yu * (uint32_t)hz), Y = (int)Yu;
            const int oct = m.oct[b], sub = m.sub[b];
            const int ix = 2 * X + ((oct >> 2) & 1), iy = 2 * Y + ((oct >> 1) & 1), iz = 2 * Z + (oct & 1);
            const uint32_t at = ((uint32_t)(ix * a.ny + iy) * (uint32_t)a.nz + (uint32_t)iz) * (uint32_t)a.nsub + sub;
            const OctSlot* ts = m.tab + b * mc;
            f3 h = {0.f, 0.f, 0.f};
            const int cn = m.cnt[b];
            for (int q = 0; q < cn; ++q) {
                const OctSlot o = ts[q];
                int jx = X + o.ex, jy = Y + o.ey, jz = Z + o.ez;
                jx += jx < 0 ? hx : 0; jx -= jx >= hx ? hx : 0;
                jy += jy < 0 ? hy : 0; jy -= jy >= hy ? hy : 0;
                jz += jz < 0 ? hz : 0; jz -= jz >= hz ? hz : 0;
                const uint32_t j = (uint32_t)o.plane + (uint32_t)((jx * hy + jy) * hz + jz);
                const f3 sj = {sx[j], sy[j], sz[j]};
                bond_term(h, sj, o);
            }
            const uint32_t si = m.base[b] + (uint32_t)X * hyz + rem;
            site_update<MOVE>(a, h, (int64_t)si, (int64_t)at, sx, sy, sz, sweep, rep, beta, de, dmx, dmy, dmz);
        }
        if (a.partials) {
            block_sum4<double>(de, dmx, dmy, dmz, tot);
            if (threadIdx.x == 0) {
                double* pp = a.partials + ((int64_t)rep * a.slots_per_rep + u) * 4;
                __stcg(pp, __ldcg(pp) + tot[0]); __stcg(pp + 1, __ldcg(pp + 1) + tot[1]);
                __stcg(pp + 2, __ldcg(pp + 2) + tot[2]); __stcg(pp + 3, __ldcg(pp + 3) + tot[3]);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            oe_st_release(e.done + r * (uint32_t)hx + u, ph + 1u);
        }
    }
}

int octant_engine_grid(int* blocks) {
    int dev = 0, sms = 0, per = 0;
    ISG_CUDA(cudaGetDevice(&dev));
    ISG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    ISG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_octant_engine<1>, kGenThreads,
                                                           (size_t)kMaxSub * 16 * sizeof(OctSlot)));
    *blocks = sms * std::max(per, 1);
    return ISING_OK;
}

int launch_octant_engine(const GeneralLaunch& a, const OctEngineLaunch& e, cudaStream_t s) {
    if (a.oct_maxcnt < 1 || e.ncls < 1 || e.n_sweeps < 1 || e.grid < 1 || e.maxnb < 1 || e.maxnb > kMaxOctBlocks)
        return fail(ISING_ERR_ARG, "octant engine setup");
    for (int c = 0; c < e.ncls; ++c)
        if (e.start[c + 1] <= e.start[c] || e.start[c + 1] - e.start[c] > e.maxnb)
            return fail(ISING_ERR_ARG, "octant engine: class list");
    OctDims od;
    od.q8 = make_div((uint32_t)a.layout.q8);
    od.hx = a.nx / 2; od.hyi = a.ny / 2; od.hzi = a.nz / 2;
    od.hz = make_div((uint32_t)od.hzi);
    od.hy = make_div((uint32_t)od.hyi);
    od.hyz = make_div((uint32_t)(od.hyi * od.hzi));
    const size_t sm = octant_smem_bytes(e.maxnb, a.oct_maxcnt);
    if (sm > 48u * 1024u) return fail(ISING_ERR_ARG, "octant engine: class stencil table exceeds 48 KB");
    if (a.move == 0) k_octant_engine<0><<<e.grid, kGenThreads, sm, s>>>(a, od, e);
    else k_octant_engine<1><<<e.grid, kGenThreads, sm, s>>>(a, od, e);
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}

// ---- sublattice classes of layout 3 (BCC without J') ------------------------------------
// A thread owns the sites z = j, j + 1 (j even) of one row (x, y) of sublattice `sub` and
// loops over rows.  Their 8 first-shell neighbours lie in the 4 rows (x + bx + a, y + by + b),
// a, b in {0, 1}, of the other sublattice, at z + bz + c, c in {0, 1}: per row one aligned
// pair (z = j, j + 1) and one edge value (j - 1 for bz = -1, j + 2 for bz = 0), so the two
// sites share their loads -- 6 component loads per row, 27 per pair of sites, with no
// per-neighbour index arithmetic.  The local field sums the bonds in (a, b, c) order with the
// stencil's expression, and each site is then updated by site_update (Philox keys of the
// reference atom index).
constexpr int kBipBlocksPerSM = 6;
int bip_slots_per_class() { return 148 * kBipBlocksPerSM; }

struct BipRow { f3 lo, hi, e; };   // z-sites j, j + 1 and the edge value of one row

template <int MOVE>
__global__ void __launch_bounds__(kGenThreads, 3) k_bip_sweep(GeneralLaunch a, BipClass bc, int sub, uint32_t rb,
                                                            uint32_t nseg, FastDiv div_seg) {
    const int rl = blockIdx.y;
    const int rep = a.rep_first + rl;
    const int64_t N = a.natoms;
    float* __restrict__ sx = a.spins + (int64_t)rl * 3 * N;
    float* __restrict__ sy = sx + N;
    float* __restrict__ sz = sy + N;
    const uint32_t sweep = a.sweep_ctr[rep] + a.sweep_offset;
    const float beta = (float)a.beta_rep[rep];
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const uint32_t lanes = (uint32_t)nz >> 1;
    const uint32_t tx = threadIdx.x % lanes, ty = threadIdx.x / lanes;
    const int j = 2 * (int)tx;
    const int oth = 1 - sub;
    const uint32_t units = (uint32_t)nx * nseg;
    const int je = bc.base[2] < 0 ? (j == 0 ? nz - 1 : j - 1) : (j + 2 == nz ? 0 : j + 2);
    auto load_row = [&](int jx, int jy) {
        const int64_t rbase = (((int64_t)oth * nx + jx) * ny + jy) * nz;
        const float2 px = *reinterpret_cast<const float2*>(sx + rbase + j);
        const float2 py = *reinterpret_cast<const float2*>(sy + rbase + j);
        const float2 pz = *reinterpret_cast<const float2*>(sz + rbase + j);
        BipRow r;
        r.lo = {px.x, py.x, pz.x};
        r.hi = {px.y, py.y, pz.y};
        r.e = {sx[rbase + je], sy[rbase + je], sz[rbase + je]};
        return r;
    };
    // bonds (a, b, c = 0, 1) of one neighbour row to the sites j and j + 1, both sites in the
    // lanes of packed FP32x2 fields (hx, hy, hz): h += w S + S x D per bond
    auto add_row = [&](const BipRow& r, int q0, float2& hx, float2& hy, float2& hz) {
        const f3 n00 = bc.base[2] < 0 ? r.e : r.lo, n01 = bc.base[2] < 0 ? r.lo : r.hi;
        const f3 n10 = bc.base[2] < 0 ? r.lo : r.hi, n11 = bc.base[2] < 0 ? r.hi : r.e;
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
            const int q = q0 + cc;
            const f3 s0 = cc ? n01 : n00, s1 = cc ? n11 : n10;
            const float2 sx_ = make_float2(s0.x, s1.x), sy_ = make_float2(s0.y, s1.y), sz_ = make_float2(s0.z, s1.z);
            const float2 w = make_float2(bc.w[q], bc.w[q]);
            const float2 Dx = make_float2(bc.D[q][0], bc.D[q][0]), Dy = make_float2(bc.D[q][1], bc.D[q][1]);
            const float2 Dz = make_float2(bc.D[q][2], bc.D[q][2]);
            const float2 nDx = make_float2(-bc.D[q][0], -bc.D[q][0]), nDy = make_float2(-bc.D[q][1], -bc.D[q][1]);
            const float2 nDz = make_float2(-bc.D[q][2], -bc.D[q][2]);
            const float2 cx = __ffma2_rn(sy_, Dz, __fmul2_rn(sz_, nDy));
            const float2 cy = __ffma2_rn(sz_, Dx, __fmul2_rn(sx_, nDz));
            const float2 cz = __ffma2_rn(sx_, Dy, __fmul2_rn(sy_, nDx));
            hx = __fadd2_rn(hx, __ffma2_rn(w, sx_, cx));
            hy = __fadd2_rn(hy, __ffma2_rn(w, sy_, cy));
            hz = __fadd2_rn(hz, __ffma2_rn(w, sz_, cz));
        }
    };
    float de = 0.f, dmx = 0.f, dmy = 0.f, dmz = 0.f;
    // a thread marches the column (x, j) of one y-segment; the row of the other sublattice at
    // y + by + 1 read for step y is the row at (y + 1) + by of the next step
#pragma unroll 1
    for (uint32_t u = ty < rb ? blockIdx.x * rb + ty : units; u < units; u += gridDim.x * rb) {
        const uint32_t ix = fdiv(u, div_seg), sg = u - ix * nseg;
        const int ya = (int)(sg * (uint32_t)ny / nseg), yb = (int)((sg + 1u) * (uint32_t)ny / nseg);
        int jx0 = (int)ix + bc.base[0], jx1 = jx0 + 1;
        jx0 += jx0 < 0 ? nx : 0; jx0 -= jx0 >= nx ? nx : 0;
        jx1 += jx1 < 0 ? nx : 0; jx1 -= jx1 >= nx ? nx : 0;
        int jy = ya + bc.base[1];
        jy += jy < 0 ? ny : 0; jy -= jy >= ny ? ny : 0;
        BipRow p0 = load_row(jx0, jy), p1 = load_row(jx1, jy);
#pragma unroll 1
        for (int iy = ya; iy < yb; ++iy) {
            jy = jy + 1 == ny ? 0 : jy + 1;
            const BipRow c0 = load_row(jx0, jy), c1 = load_row(jx1, jy);
            float2 hx = make_float2(0.f, 0.f), hy = hx, hz = hx;
            add_row(p0, 0, hx, hy, hz);   // (a, b) = (0, 0)
            add_row(c0, 2, hx, hy, hz);   // (0, 1)
            add_row(p1, 4, hx, hy, hz);   // (1, 0)
            add_row(c1, 6, hx, hy, hz);   // (1, 1)
            p0 = c0;
            p1 = c1;
            const int64_t own = (((int64_t)sub * nx + ix) * ny + iy) * nz + j;
            const uint32_t at = (uint32_t)((((int64_t)ix * ny + iy) * nz + j) * 2 + sub);
            site_update_pair<MOVE>(a, hx, hy, hz, own, at, at + 2u, sx, sy, sz, sweep, rep, beta, de, dmx, dmy, dmz);
        }
    }
    if (a.partials) {
        __shared__ double tot[4];
        block_sum4_fd(de, dmx, dmy, dmz, tot);
        if (threadIdx.x == 0) {
            double* p = a.partials + ((int64_t)rep * a.slots_per_rep + a.slot_base + blockIdx.x) * 4;
            p[0] += tot[0]; p[1] += tot[1]; p[2] += tot[2]; p[3] += tot[3];
        }
    }
}

int launch_bip_sweep(const GeneralLaunch& a, const BipClass& c, int sub, cudaStream_t s) {
    if (a.n_rep <= 0) return ISING_OK;
    if (a.nsub != 2 || sub < 0 || sub > 1 || a.nz % 2 || a.nz / 2 > kGenThreads || a.layout.cb != 3)
        return fail(ISING_ERR_ARG, "sublattice-class sweep needs layout 3 and an even nz <= 512");
    const uint32_t lanes = (uint32_t)(a.nz / 2), rb = std::max(1u, (uint32_t)kGenThreads / lanes);
    // y-segments per x-column: enough column units for about two blocks of work per resident
    // block slot, every segment at least two rows long
    const int64_t want_units = 2LL * bip_slots_per_class() * rb;
    int64_t nseg = (want_units + (int64_t)a.nx * a.n_rep - 1) / ((int64_t)a.nx * a.n_rep);
    nseg = std::max<int64_t>(1, std::min<int64_t>(nseg, a.ny / 2));
    const uint32_t units = (uint32_t)(a.nx * nseg);
    int zb = (int)((units + rb - 1) / rb);
    zb = std::max(1, std::min(zb, bip_slots_per_class()));
    dim3 g(zb, a.n_rep), b(kGenThreads);
    const FastDiv dseg = make_div((uint32_t)nseg);
    if (a.move == 0) k_bip_sweep<0><<<g, b, 0, s>>>(a, c, sub, rb, (uint32_t)nseg, dseg);
    else k_bip_sweep<1><<<g, b, 0, s>>>(a, c, sub, rb, (uint32_t)nseg, dseg);
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}

int octant_slots_for(int64_t n_sites, bool fast) {
    const int64_t per = (int64_t)kGenThreads * (fast ? 1 : kGenSitesPerThread);
    return (int)((n_sites + per - 1) / per);
}

// blocks of one class launch: as many as keep the block stencils within 48 KB of shared memory
static int octant_chunk(int maxcnt) {
    if (maxcnt < 1) return 1;   // k_octant_colour: one launch per block
    const int fit = (int)((48u * 1024u) / octant_smem_bytes(1, maxcnt));
    return std::max(1, std::min(kMaxOctBlocks, fit));
}

int octant_class_launches(int nblocks, int maxcnt) {
    const int c = octant_chunk(maxcnt);
    return (nblocks + c - 1) / c;
}

int octant_class_slots(int64_t q8, int nblocks, int maxcnt) {
    const int c = octant_chunk(maxcnt);
    int tot = 0;
    for (int b0 = 0; b0 < nblocks; b0 += c) tot += octant_slots_for(q8 * std::min(c, nblocks - b0), maxcnt > 0);
    return tot;
}

int launch_octant_class(const GeneralLaunch& a, const OctBlocks& bl, cudaStream_t s) {
    if (bl.n < 1 || bl.n > kMaxOctBlocks) return fail(ISING_ERR_ARG, "octant class: 1 to 128 blocks");
    for (int k = 0; k < bl.n; ++k)
        if ((bl.code[k] & 15) >= a.nsub) return fail(ISING_ERR_ARG, "octant class block out of range");
    const int64_t q8 = a.layout.q8;
    const int chunk = octant_chunk(a.oct_maxcnt);
    if (bl.n > chunk) {   // consecutive runs of blocks, one launch each (the class's sites are independent)
        GeneralLaunch g = a;
        for (int b0 = 0; b0 < bl.n; b0 += chunk) {
            OctBlocks part{};
            part.n = std::min(chunk, bl.n - b0);
            for (int k = 0; k < part.n; ++k) part.code[k] = bl.code[b0 + k];
            const int rc = launch_octant_class(g, part, s);
            if (rc != ISING_OK) return rc;
            g.slot_base += octant_slots_for(q8 * part.n, a.oct_maxcnt > 0);
        }
        return ISING_OK;
    }
    dim3 b(kGenThreads);
    if (a.oct_maxcnt < 1) {   // a single block: the cell-coordinate stencil
        dim3 g(octant_slots_for(q8, false), a.n_rep);
        const size_t sm = (size_t)a.st.nsub * kMaxSlots * sizeof(Slot) + kMaxSub * sizeof(int);
        const int oct = bl.code[0] >> 4, rank = bl.code[0] & 15;
        if (a.move == 0) k_octant_colour<0><<<g, b, sm, s>>>(a, oct, rank, 1);
        else k_octant_colour<1><<<g, b, sm, s>>>(a, oct, rank, 1);
        ISG_CUDA(cudaGetLastError());
        return ISING_OK;
    }
    // sites (pairs) per thread: as many as keep about two waves of blocks (6 resident per SM);
    // fewer blocks than partial slots leave the last slots at zero
    int sms = 148;
    {
        int dev = 0;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    const int64_t ntot = q8 * bl.n;
    const int64_t per_launch = ntot * a.n_rep, want = 2LL * sms * 6 * kGenThreads;
    OctDims od;
    od.q8 = make_div((uint32_t)q8);
    od.hx = a.nx / 2; od.hyi = a.ny / 2; od.hzi = a.nz / 2;
    od.hz = make_div((uint32_t)od.hzi);
    od.hy = make_div((uint32_t)od.hyi);
    const size_t sm = octant_smem_bytes(bl.n, a.oct_maxcnt);
    if (od.hzi % 2 == 0) {   // site pairs along packed z (q8 is even)
        od.q8h = make_div((uint32_t)(q8 / 2));
        const int ppt = per_launch / 2 >= 4 * want ? 4 : (per_launch / 2 >= 2 * want ? 2 : 1);
        // <= octant_slots_for(ntot, true) blocks
        dim3 g((unsigned)((ntot / 2 + (int64_t)kGenThreads * ppt - 1) / ((int64_t)kGenThreads * ppt)), a.n_rep);
#define ISG_OP(P)                                                          \
    if (a.move == 0) k_octant_pair<0, P><<<g, b, sm, s>>>(a, od, bl);      \
    else k_octant_pair<1, P><<<g, b, sm, s>>>(a, od, bl);
        if (ppt == 4) { ISG_OP(4) } else if (ppt == 2) { ISG_OP(2) } else { ISG_OP(1) }
#undef ISG_OP
        ISG_CUDA(cudaGetLastError());
        return ISING_OK;
    }
    const int spt = per_launch >= 4 * want ? 4 : (per_launch >= 2 * want ? 2 : 1);
    dim3 g((unsigned)((ntot + (int64_t)kGenThreads * spt - 1) / ((int64_t)kGenThreads * spt)), a.n_rep);
#define ISG_OF(S)                                                          \
    if (a.move == 0) k_octant_fast<0, S><<<g, b, sm, s>>>(a, od, bl);      \
    else k_octant_fast<1, S><<<g, b, sm, s>>>(a, od, bl);
    if (spt == 4) { ISG_OF(4) } else if (spt == 2) { ISG_OF(2) } else { ISG_OF(1) }
#undef ISG_OF
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}

int launch_general_colour(const GeneralLaunch& a, cudaStream_t s) {
    if (a.n_sites <= 0) return ISING_OK;
    dim3 g(general_slots_for(a.n_sites), a.n_rep), b(kGenThreads);
    size_t sm = (size_t)a.st.nsub * kMaxSlots * sizeof(Slot) + kMaxSub * sizeof(int);
    if (a.move == 0) k_general_colour<0><<<g, b, sm, s>>>(a);
    else k_general_colour<1><<<g, b, sm, s>>>(a);
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}

// ================================================================= energy + magnetisation
// e_i = 1/2 S.(sum_j w S_j + S_j x D_ij) - Bz S_z - K (S.e)^2, summed per replica:
// TotalHeisenbergEnergy (src/energyMin.f90:499-528) with FP32 terms and FP64 block sums.
constexpr int kRedThreads = 256;
constexpr int kRedSitesPerBlock = 4096;

int energy_blocks_for(int64_t natoms) {
    return (int)((natoms + kRedSitesPerBlock - 1) / kRedSitesPerBlock);
}

__global__ void __launch_bounds__(kRedThreads) k_energy_mag(ReduceLaunch a) {
    extern __shared__ unsigned char smem_raw[];
    Slot* sl = reinterpret_cast<Slot*>(smem_raw);
    int* cnt = reinterpret_cast<int*>(sl + a.st.nsub * kMaxSlots);
    for (int q = threadIdx.x; q < a.st.nsub * kMaxSlots; q += blockDim.x) sl[q] = a.st.slots[q];
    for (int q = threadIdx.x; q < a.st.nsub; q += blockDim.x) cnt[q] = a.st.count[q];
    __syncthreads();
    const int rep = blockIdx.y;
    const int64_t N = a.natoms;
    const float* sx = a.spins + (int64_t)rep * 3 * N;
    const float* sy = sx + N;
    const float* sz = sy + N;
    const HamDev& H = a.ham;
    double e = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
    const int64_t i0 = (int64_t)blockIdx.x * kRedSitesPerBlock;
    int64_t i1 = i0 + kRedSitesPerBlock;
    if (i1 > N) i1 = N;
    for (int64_t at = i0 + threadIdx.x; at < i1; at += blockDim.x) {
        int ix, iy, iz, sub;
        decode_atom(at, a.nsub, a.ny, a.nz, &ix, &iy, &iz, &sub);
        const f3 h = stencil_field(sx, sy, sz, sl + sub * kMaxSlots, cnt[sub], ix, iy, iz, a.layout);
        const int64_t si = sidx(a.layout, ix, iy, iz, sub);
        const f3 s = {sx[si], sy[si], sz[si]};
        float ei = 0.5f * dot(s, h) - H.Bz * s.z;
        if (H.K != 0.f) {
            const float ea = s.x * H.kx + s.y * H.ky + s.z * H.kz;
            ei -= H.K * ea * ea;
        }
        e += (double)ei;
        mx += (double)s.x; my += (double)s.y; mz += (double)s.z;
    }
    __shared__ double tot[4];
    block_sum4<double>(e, mx, my, mz, tot);
    if (threadIdx.x == 0) {
        double* p = a.block_tmp + ((int64_t)rep * a.blocks_per_rep + blockIdx.x) * 4;
        p[0] = tot[0]; p[1] = tot[1]; p[2] = tot[2]; p[3] = tot[3];
    }
}

// Deterministic per-replica sum of block partials: out[rep] = sum_b in[rep][b]; optionally
// accumulate into acc and zero the inputs.
__global__ void k_sum_blocks(double* in, int nb, double* out, Acc4* acc, int zero_in) {
    const int rep = blockIdx.x;
    double v[4] = {0, 0, 0, 0};
    double* p = in + (int64_t)rep * nb * 4;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        for (int q = 0; q < 4; ++q) v[q] += p[(int64_t)b * 4 + q];
        if (zero_in) for (int q = 0; q < 4; ++q) p[(int64_t)b * 4 + q] = 0.0;
    }
    __shared__ double tot[4];
    block_sum4<double>(v[0], v[1], v[2], v[3], tot);
    if (threadIdx.x == 0) {
        if (out) for (int q = 0; q < 4; ++q) out[rep * 4 + q] = tot[q];
        if (acc) { acc[rep].e += tot[0]; acc[rep].mx += tot[1]; acc[rep].my += tot[2]; acc[rep].mz += tot[3]; }
    }
}

int launch_energy_mag(const ReduceLaunch& a, cudaStream_t s) {
    dim3 g(a.blocks_per_rep, a.n_rep);
    size_t sm = (size_t)a.st.nsub * kMaxSlots * sizeof(Slot) + kMaxSub * sizeof(int);
    k_energy_mag<<<g, kRedThreads, sm, s>>>(a);
    ISG_CUDA(cudaGetLastError());
    k_sum_blocks<<<a.n_rep, 256, 0, s>>>(a.block_tmp, a.blocks_per_rep, a.out, nullptr, 0);
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}

int launch_fold_partials(double* partials, int slots_per_rep, int n_rep, Acc4* acc, cudaStream_t s) {
    k_sum_blocks<<<n_rep, 256, 0, s>>>(partials, slots_per_rep, nullptr, acc, 1);
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}

// ================================================================= winding number
// Per z-slice Berg-Luscher topological charge (calculate_winding_number2, rsp:320-364 with
// arc_winding rsp:284-318): plaquette (s1, s1+a, s1+b, s1+a+b) from the derivative list,
// triangles (s1,s2,s4) and (s1,s4,s3), divided by 4*pi (pi as the reference's
// default-real literal).
// One block per (slice, replica). With a.dens set, every plaquette also stores its density
// (calculate_winding_number_density, rsp:438-500): density_matrix(i,j) column-major per slice,
// which the x-fastest plaquette order writes coalesced.
template <typename T>
__global__ void __launch_bounds__(256) k_winding(WindingLaunch a) {
    const int zc = a.z0 + blockIdx.x;
    const int rep = blockIdx.y;
    const int64_t N = a.natoms;
    const float* sx = a.spins + (int64_t)rep * 3 * N;
    const float* sy = sx + N;
    const float* sz = sy + N;
    const int* P = a.plaq;  // 4 x (dx, dy, dz, sub): s1, s2, s4, s3
    T w = T(0);
    const int np = a.nx * a.ny;
    double* dn = a.dens ? a.dens + ((int64_t)rep * gridDim.x + blockIdx.x) * np : nullptr;
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
        const int i = p % a.nx, j = p / a.nx;
        int64_t at[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int jx = wrap_any(i + P[4 * q], a.nx), jy = wrap_any(j + P[4 * q + 1], a.ny);
            const int jz = wrap_any(zc + P[4 * q + 2], a.nz);
            at[q] = sidx(a.layout, jx, jy, jz, P[4 * q + 3]);
        }
        T s1[3], s2[3], s4[3], s3[3];
        load_unit<T>(sx, sy, sz, at[0], s1);
        load_unit<T>(sx, sy, sz, at[1], s2);
        load_unit<T>(sx, sy, sz, at[2], s4);
        load_unit<T>(sx, sy, sz, at[3], s3);
        const T pl = arc_winding_t<T>(s1, s2, s4) + arc_winding_t<T>(s1, s4, s3);
        w += pl;
        if (dn) dn[p] = (double)pl / (4.0 * (double)3.14159265358979323846f);
    }
    __shared__ double tot[4];
    block_sum4<double>((double)w, 0.0, 0.0, 0.0, tot);
    if (threadIdx.x == 0) {
        const double four_pi = 4.0 * (double)3.14159265358979323846f;
        a.out[(int64_t)rep * a.nz + zc] = tot[0] / four_pi;
    }
}

int launch_winding(const WindingLaunch& a, cudaStream_t s) {
    const int nzc = a.nzc > 0 ? a.nzc : a.nz;
    if (a.z0 < 0 || a.z0 + nzc > a.nz) return fail(ISING_ERR_BOUNDS, "winding slice range out of bounds");
    dim3 g(nzc, a.n_rep);
    if (a.fp64) k_winding<double><<<g, 256, 0, s>>>(a);
    else k_winding<float><<<g, 256, 0, s>>>(a);
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}

// ================================================================= local energy queries
// calculateHeisenbergEnergy (src/energyMin.f90:86-171) for a batch of (atom, S') pairs:
// E(S) = S.h - K (S.e)^2 with h the FP32 local field.
__global__ void k_local_energy(LocalLaunch a) {
    extern __shared__ unsigned char smem_raw[];
    Slot* sl = reinterpret_cast<Slot*>(smem_raw);
    int* cnt = reinterpret_cast<int*>(sl + a.st.nsub * kMaxSlots);
    for (int q = threadIdx.x; q < a.st.nsub * kMaxSlots; q += blockDim.x) sl[q] = a.st.slots[q];
    for (int q = threadIdx.x; q < a.st.nsub; q += blockDim.x) cnt[q] = a.st.count[q];
    __syncthreads();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.n) return;
    const int64_t N = a.natoms;
    const float* sx = a.spins;
    const float* sy = sx + N;
    const float* sz = sy + N;
    const int64_t at = a.atoms[t];
    int ix, iy, iz, sub;
    decode_atom(at, a.nsub, a.ny, a.nz, &ix, &iy, &iz, &sub);
    f3 h = stencil_field(sx, sy, sz, sl + sub * kMaxSlots, cnt[sub], ix, iy, iz, a.layout);
    h.z -= a.ham.Bz;
    const int64_t si = sidx(a.layout, ix, iy, iz, sub);
    const f3 s = {sx[si], sy[si], sz[si]};
    const f3 sp = {(float)a.sprop[3 * t], (float)a.sprop[3 * t + 1], (float)a.sprop[3 * t + 2]};
    float e0 = dot(s, h), e1 = dot(sp, h);
    if (a.ham.K != 0.f) {
        const float q0 = s.x * a.ham.kx + s.y * a.ham.ky + s.z * a.ham.kz;
        const float q1 = sp.x * a.ham.kx + sp.y * a.ham.ky + sp.z * a.ham.kz;
        e0 -= a.ham.K * q0 * q0;
        e1 -= a.ham.K * q1 * q1;
    }
    if (a.demag_H) {   // -mu_0 S.H in FP64 (src/energyMin.f90:163-167)
        const double hx = a.demag_H[at], hy = a.demag_H[N + at], hz = a.demag_H[2 * N + at];
        a.old_e[t] = (double)e0 - kMu0 * ((double)s.x * hx + (double)s.y * hy + (double)s.z * hz);
        a.new_e[t] = (double)e1 - kMu0 * (a.sprop[3 * t] * hx + a.sprop[3 * t + 1] * hy + a.sprop[3 * t + 2] * hz);
        return;
    }
    a.old_e[t] = (double)e0;
    a.new_e[t] = (double)e1;
}

int launch_local_energy(const LocalLaunch& a, cudaStream_t s) {
    if (a.n <= 0) return ISING_OK;
    size_t sm = (size_t)a.st.nsub * kMaxSlots * sizeof(Slot) + kMaxSub * sizeof(int);
    k_local_energy<<<(a.n + 127) / 128, 128, sm, s>>>(a);
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}

// ================================================================= initial spins
__global__ void k_init_uniform(float* spins, int64_t N, Layout L, uint64_t seed, uint32_t ensemble) {
    const int rep = blockIdx.y;
    float* sx = spins + (int64_t)rep * 3 * N;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const uint4 r4 = philox4x32<10>(make_uint4((uint32_t)i, 0u, (uint32_t)rep, (ensemble << 8) | kTagInit),
                                        philox_key(seed));
        // uniform unit vector: cos theta = 2u-1, azimuth 2 pi (u - 1/2), normalised
        const float cz = fmaf(2.0f, u01(r4.x), -1.0f);
        const float st = sqrtf(fmaf(-cz, cz, 1.0f));
        float sn, cs;
        sincospif(2.0f * (u01(r4.y) - 0.5f), &sn, &cs);
        f3 v = {st * cs, st * sn, cz};
        const float rn = rsqrtf(dot(v, v));
        const int64_t j = sidx_atom(L, i);
        sx[j] = v.x * rn; sx[N + j] = v.y * rn; sx[2 * N + j] = v.z * rn;
    }
}

int launch_init_uniform(float* spins, int64_t natoms, const Layout& L, int n_rep, uint64_t seed,
                        uint32_t ensemble, cudaStream_t s) {
    int blocks = (int)((natoms + 255) / 256);
    if (blocks > 4096) blocks = 4096;
    dim3 g(blocks, n_rep);
    k_init_uniform<<<g, 256, 0, s>>>(spins, natoms, L, seed, ensemble);
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}

__global__ void k_advance(uint32_t* ctr, int n, uint32_t by) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) ctr[i] += by;
}

int launch_advance(uint32_t* ctr, int n, uint32_t by, cudaStream_t s) {
    k_advance<<<(n + 255) / 256, 256, 0, s>>>(ctr, n, by);
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}

// ================================================================= replica exchange
// One exchange round (exchange.cuh) as its own single-block launch.
__global__ void k_exchange(ExchangeLaunch a) { exchange_round(a); }

int launch_exchange(const ExchangeLaunch& a, cudaStream_t s) {
    if (a.n < 2) return ISING_OK;
    k_exchange<<<1, 256, 0, s>>>(a);
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}

// ================================================================= per-sweep record
// One row per temperature slot t: observables of the replica that holds slot t now.
__global__ void k_record(RecordLaunch a) {
    const int c = *a.count;
    if (c < a.cap) {
        for (int t = threadIdx.x; t < a.n_rep; t += blockDim.x) {
            const int rep = a.t2r[t];
            const Acc4 v = a.acc[rep];
            double* o = a.series + ((int64_t)t * a.cap + c) * 4;
            const double m = sqrt(v.mx * v.mx + v.my * v.my + v.mz * v.mz) / (double)a.natoms;
            double qs = 0.0;
            for (int z = 0; z < a.nz; ++z) qs += a.q[(int64_t)rep * a.nz + z];
            const int zmid = a.nz / 2 - 1 >= 0 ? a.nz / 2 - 1 : 0;  // winding_array(numCellsZ/2)
            o[0] = v.e;
            o[1] = m;
            o[2] = a.q[(int64_t)rep * a.nz + zmid];
            o[3] = qs / (double)a.nz;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && c < a.cap) *a.count = c + 1;
}

int launch_record(const RecordLaunch& a, cudaStream_t s) {
    k_record<<<1, 256, 0, s>>>(a);
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}

// ================================================================= host-layout conversion
// atomSpins(numAtoms,3) column-major FP64 is the planes layout already; only the width
// changes.  Zero or non-finite vectors raise the NaN status (src/energyMin.f90:330-331).
__global__ void k_spins_from_f64(const double* in, float* out, int64_t N, Layout L, int* status) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const double x = in[i], y = in[N + i], z = in[2 * N + i];
        const double n2 = x * x + y * y + z * z;
        if (!(n2 > 0.0) || !isfinite(n2)) atomicOr(status, kStatNan);
        const int64_t j = sidx_atom(L, i);
        out[j] = (float)x; out[N + j] = (float)y; out[2 * N + j] = (float)z;
    }
}

__global__ void k_spins_to_f64(const float* in, double* out, int64_t N, Layout L) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = sidx_atom(L, i);
        out[i] = (double)in[j]; out[N + i] = (double)in[N + j]; out[2 * N + i] = (double)in[2 * N + j];
    }
}

int launch_spins_from_f64(const double* in, float* out, int64_t natoms, const Layout& L, int* status,
                          cudaStream_t s) {
    int blocks = (int)((natoms + 255) / 256);
    if (blocks > 8192) blocks = 8192;
    k_spins_from_f64<<<blocks, 256, 0, s>>>(in, out, natoms, L, status);
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}

int launch_spins_to_f64(const float* in, double* out, int64_t natoms, const Layout& L, cudaStream_t s) {
    int blocks = (int)((natoms + 255) / 256);
    if (blocks > 8192) blocks = 8192;
    k_spins_to_f64<<<blocks, 256, 0, s>>>(in, out, natoms, L);
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}

}  // namespace isg
