// sweep_cb.cuh -- device code shared by the checkerboard sweep kernels (one launch per colour
// pass in sweep_cb.cu, the persistent multi-ensemble engine in ensembles.cu).
//
// Storage: per replica and spin component, the N/2 sites of colour 0 then those of colour 1;
// inside a colour, packed rows of W = nz/2 entries in (x, y) order, entry j of row (x, y)
// being the site z = 2j + ((x + y + colour) & 1).  A thread owns a pair of consecutive
// entries (j, j+1) of one packed row and updates both sites in lockstep with the packed
// FP32x2 arithmetic of sm_100 (__ffma2_rn / __fadd2_rn / __fmul2_rn): lane .x is the site
// z0 = 2j + p, lane .y the site z0 + 2.  All six neighbours of a site have the other colour:
// the x/y neighbours are the pair (j, j+1) of the rows (x+-1, y), (x, y+-1); the z
// neighbours are entries j-1..j+2 of the other colour's row (x, y).
//
// The local field and dE follow calculateHeisenbergEnergy (reference
// src/energyMin.f90:86-171) in local-field form: h = J sum S_j + sum_k S_k x D_k - B z_hat,
// dE = (S' - S).h - K[(S'.e)^2 - (S.e)^2].
#pragma once
#include "internal.h"

namespace isg {

using v2 = float2;
__device__ __forceinline__ v2 V(float a) { return make_float2(a, a); }
__device__ __forceinline__ v2 add(v2 a, v2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ v2 sub(v2 a, v2 b) { return __ffma2_rn(b, V(-1.f), a); }
__device__ __forceinline__ v2 mul(v2 a, v2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ v2 fma2(v2 a, v2 b, v2 c) { return __ffma2_rn(a, b, c); }

struct v23 { v2 x, y, z; };   // a pair of 3-vectors, component-major

__device__ __forceinline__ v23 ld3(const float* sx, const float* sy, const float* sz, uint32_t o) {
    return {*reinterpret_cast<const v2*>(sx + o), *reinterpret_cast<const v2*>(sy + o),
            *reinterpret_cast<const v2*>(sz + o)};
}


// Geometry and Hamiltonian of one colour-separated simple-cubic mesh, as the pair update
// reads them.
struct CbGeom {
    HamDev ham;
    int nx, ny, nz;
    uint32_t W;             // packed row length nz/2
    uint32_t half;          // N/2
    uint32_t row_stride_x;  // W * ny: packed entries per x-plane
    uint32_t ensemble;
    float r;                // ball-step radius
};

// The two Philox draws of the site pair (j, j+1) of packed row `row` (parity p): counters
// (reference atom index, sweep, replica, ensemble << 8 | sweep tag).
__device__ __forceinline__ void pair_draws(const CbGeom& P, const uint32_t* rk, uint32_t row, uint32_t j,
                                           uint32_t p, uint32_t sweep, uint32_t rep, uint4& ra, uint4& rb) {
    const uint32_t i0 = row * (uint32_t)P.nz + 2u * j + p;   // reference atom index of site .x
    const uint32_t cw = (P.ensemble << 8) | kTagSweep;
    ra = philox_rk(make_uint4(i0, sweep, rep, cw), rk);
    rb = philox_rk(make_uint4(i0 + 2u, sweep, rep, cw), rk);
}

// Update of one site pair from its loaded neighbourhood: own pair s at entries (j, j+1) of
// packed row `row` (parity p), the other colour's pairs px, mx (x +- 1), py, my (y +- 1) and
// oz (same row) at entries (j, j+1), and the edge entry (ex, ey, ez) of that row.  Returns
// the pair after the Metropolis decisions (rejected sites bit-identical to s); `any` tells
// whether either site accepted.  dE and dM of accepted moves are added to the running sums
// when `count` is set (a recomputed halo pair is not counted).
// pair_new_drawn takes the pair's Philox draws (pair_draws); pair_new draws them itself.
template <int MOVE, int DMI, bool HAS_K>
__device__ __forceinline__ v23 pair_new_drawn(const CbGeom& P, int* status, uint32_t p, const v23& s,
                                              const v23& px, const v23& mx, const v23& py, const v23& my,
                                              const v23& oz, float ex, float ey, float ez, const uint4& ra,
                                              const uint4& rb, float beta2, bool count, v2& de, v2& dmx, v2& dmy,
                                              v2& dmz, bool& any) {
    const CbGeom& a = P;
    const HamDev& H = P.ham;
    v23 zp, zm;
    if (p) {   // site z = 2j+1(+2): z+1 -> j+1 (j+2), z-1 -> j (j+1)
        zp = {make_float2(oz.x.y, ex), make_float2(oz.y.y, ey), make_float2(oz.z.y, ez)};
        zm = oz;
    } else {   // site z = 2j(+2): z+1 -> j (j+1), z-1 -> j-1 (j)
        zp = oz;
        zm = {make_float2(ex, oz.x.x), make_float2(ey, oz.y.x), make_float2(ez, oz.z.x)};
    }
    // local field for both sites
    const v2 J = V(H.J);
    v23 h;
    h.x = mul(J, add(add(add(px.x, mx.x), add(py.x, my.x)), add(zp.x, zm.x)));
    h.y = mul(J, add(add(add(px.y, mx.y), add(py.y, my.y)), add(zp.y, zm.y)));
    h.z = mul(J, add(add(add(px.z, mx.z), add(py.z, my.z)), add(zp.z, zm.z)));
    if (DMI == 1) {        // bulk: D (S_{-a} - S_{+a}) x a_hat
        const v2 D = V(H.D[1][0]);
        h.x = fma2(D, sub(sub(zm.y, zp.y), sub(my.z, py.z)), h.x);
        h.y = fma2(D, sub(sub(mx.z, px.z), sub(zm.x, zp.x)), h.y);
        h.z = fma2(D, sub(sub(my.x, py.x), sub(mx.y, px.y)), h.z);
    } else if (DMI == 2) { // interfacial about z
        const v2 D = V(H.D[2][0]);
        h.x = fma2(D, sub(px.z, mx.z), h.x);
        h.y = fma2(D, sub(py.z, my.z), h.y);
        h.z = fma2(D, sub(sub(mx.x, px.x), sub(py.y, my.y)), h.z);
    } else if (DMI == 3) { // tabulated D per direction: h += n x D_k
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

    // packed proposals from the draws
    v23 sp;
    {
        const float2 sv[3] = {s.x, s.y, s.z};
        float2 o[3];
        propose2<MOVE>(sv, ra, rb, a.r, o);
        sp = {o[0], o[1], o[2]};
    }
    const v23 d = {sub(sp.x, s.x), sub(sp.y, s.y), sub(sp.z, s.z)};
    v2 dE = fma2(d.x, h.x, fma2(d.y, h.y, mul(d.z, h.z)));
    if (HAS_K) {
        const v2 e1 = fma2(sp.x, V(H.kx), fma2(sp.y, V(H.ky), mul(sp.z, V(H.kz))));
        const v2 e0 = fma2(s.x, V(H.kx), fma2(s.y, V(H.ky), mul(s.z, V(H.kz))));
        dE = fma2(V(-H.K), mul(sub(e1, e0), add(e1, e0)), dE);
    }
    if (!(dE.x == dE.x) || !(dE.y == dE.y)) atomicOr(status, kStatNan);
    // beta2 = beta * log2(e): exp(-beta dE) = 2^(-beta2 dE)
    const v2 t = mul(V(-beta2), dE);
    const v2 u3 = add(make_float2(__uint_as_float((ra.w >> 9) | 0x3f800000u), __uint_as_float((rb.w >> 9) | 0x3f800000u)),
                      V(-0.99999994f));
    const bool acc0 = (dE.x <= 0.f) || (u3.x < ax_ex2(t.x));
    const bool acc1 = (dE.y <= 0.f) || (u3.y < ax_ex2(t.y));
    if (count) {
        const v2 m = make_float2(acc0 ? 1.f : 0.f, acc1 ? 1.f : 0.f);
        de = fma2(m, dE, de);
        dmx = fma2(m, d.x, dmx);
        dmy = fma2(m, d.y, dmy);
        dmz = fma2(m, d.z, dmz);
    }
    // rejected sites keep s bit for bit, accepted ones take S' exactly
    any = acc0 | acc1;
    return {make_float2(acc0 ? sp.x.x : s.x.x, acc1 ? sp.x.y : s.x.y),
            make_float2(acc0 ? sp.y.x : s.y.x, acc1 ? sp.y.y : s.y.y),
            make_float2(acc0 ? sp.z.x : s.z.x, acc1 ? sp.z.y : s.z.y)};
}

template <int MOVE, int DMI, bool HAS_K>
__device__ __forceinline__ v23 pair_new(const CbGeom& P, const uint32_t* rk, int* status, uint32_t row,
                                        uint32_t j, uint32_t p, const v23& s, const v23& px, const v23& mx,
                                        const v23& py, const v23& my, const v23& oz, float ex, float ey,
                                        float ez, uint32_t sweep, uint32_t rep, float beta2, bool count,
                                        v2& de, v2& dmx, v2& dmy, v2& dmz, bool& any) {
    uint4 ra, rb;
    pair_draws(P, rk, row, j, p, sweep, rep, ra, rb);
    return pair_new_drawn<MOVE, DMI, HAS_K>(P, status, p, s, px, mx, py, my, oz, ex, ey, ez, ra, rb, beta2, count,
                                            de, dmx, dmy, dmz, any);
}

// pair_new, with the pair written back at own_off when either site accepts.
template <int MOVE, int DMI, bool HAS_K>
__device__ __forceinline__ void pair_compute(const CbGeom& P, const uint32_t* rk, int* status,
                                             float* __restrict__ sx, float* __restrict__ sy,
                                             float* __restrict__ sz, uint32_t own_off, uint32_t row,
                                             uint32_t j, uint32_t p, const v23& s, const v23& px, const v23& mx,
                                             const v23& py, const v23& my, const v23& oz, float ex, float ey,
                                             float ez, uint32_t sweep, uint32_t rep, float beta2,
                                             v2& de, v2& dmx, v2& dmy, v2& dmz) {
    bool any;
    const v23 n = pair_new<MOVE, DMI, HAS_K>(P, rk, status, row, j, p, s, px, mx, py, my, oz, ex, ey, ez, sweep,
                                             rep, beta2, true, de, dmx, dmy, dmz, any);
    if (any) {
        *reinterpret_cast<v2*>(sx + own_off) = n.x;
        *reinterpret_cast<v2*>(sy + own_off) = n.y;
        *reinterpret_cast<v2*>(sz + own_off) = n.z;
    }
}

template <int MOVE, int DMI, bool HAS_K>
__device__ __forceinline__ void pair_update(const CbGeom& P, const uint32_t* rk, int* status,
                                            float* __restrict__ sx, float* __restrict__ sy,
                                            float* __restrict__ sz, uint32_t row, uint32_t x, uint32_t y,
                                            uint32_t j, int colour, uint32_t sweep, uint32_t rep, float beta2,
                                            v2& de, v2& dmx, v2& dmy, v2& dmz) {
    const CbGeom& a = P;
    const uint32_t p = (x + y + (uint32_t)colour) & 1u;
    const uint32_t own = (uint32_t)colour * P.half;
    const uint32_t oth = (uint32_t)(colour ^ 1) * P.half;
    const uint32_t rowW = row * P.W;
    // neighbour rows of the other colour
    const uint32_t xs = P.row_stride_x;
    const uint32_t r_xp = x + 1 == (uint32_t)a.nx ? rowW - x * xs : rowW + xs;
    const uint32_t r_xm = x == 0 ? rowW + ((uint32_t)a.nx - 1) * xs : rowW - xs;
    const uint32_t r_yp = y + 1 == (uint32_t)a.ny ? rowW - y * P.W : rowW + P.W;
    const uint32_t r_ym = y == 0 ? rowW + ((uint32_t)a.ny - 1) * P.W : rowW - P.W;

    v23 s = ld3(sx, sy, sz, own + rowW + j);
    const v23 px = ld3(sx, sy, sz, oth + r_xp + j);
    const v23 mx = ld3(sx, sy, sz, oth + r_xm + j);
    const v23 py = ld3(sx, sy, sz, oth + r_yp + j);
    const v23 my = ld3(sx, sy, sz, oth + r_ym + j);
    const v23 oz = ld3(sx, sy, sz, oth + rowW + j);
    // edge entry of the other colour's row: j-1 (p = 0) or j+2 (p = 1), periodic in the row
    const uint32_t je = p ? (j + 2 == P.W ? 0u : j + 2) : (j == 0 ? P.W - 1 : j - 1);
    const uint32_t oe = oth + rowW + je;
    const float ex = sx[oe], ey = sy[oe], ez = sz[oe];
    pair_compute<MOVE, DMI, HAS_K>(P, rk, status, sx, sy, sz, own + rowW + j, row, j, p, s, px, mx, py, my, oz,
                                   ex, ey, ez, sweep, rep, beta2, de, dmx, dmy, dmz);
}


// One thread's march along y over rows [ya, yb) of x-plane x at entry pair (j, j+1): the
// other colour's row (x, y+1) loaded for row y is also the z-neighbour row of y+1 and the
// (y-1)-row of y+2, so a pair costs 15 loads (own pair, y+1 row, x +- 1 rows, one edge entry)
// instead of 21.
template <int MOVE, int DMI, bool HAS_K>
__device__ __forceinline__ void march_column(const CbGeom& G, const uint32_t* rk, int* status,
                                             float* __restrict__ sx, float* __restrict__ sy,
                                             float* __restrict__ sz, uint32_t x, uint32_t ya, uint32_t yb,
                                             uint32_t j, int colour, uint32_t sweep, uint32_t rep, float beta2,
                                             v2& de, v2& dmx, v2& dmy, v2& dmz) {
    const uint32_t ny = (uint32_t)G.ny, nx = (uint32_t)G.nx, W = G.W, xs = G.row_stride_x;
    const uint32_t own = (uint32_t)colour * G.half, oth = (uint32_t)(colour ^ 1) * G.half;
    const uint32_t pl = x * xs;
    const uint32_t plp = x + 1 == nx ? 0u : pl + xs;
    const uint32_t plm = x == 0 ? (nx - 1) * xs : pl - xs;
    v23 prev = ld3(sx, sy, sz, oth + pl + (ya == 0 ? ny - 1 : ya - 1) * W + j);
    v23 cur = ld3(sx, sy, sz, oth + pl + ya * W + j);
#pragma unroll 1
    for (uint32_t y = ya; y < yb; ++y) {
        const uint32_t rw = y * W;
        const v23 next = ld3(sx, sy, sz, oth + pl + (y + 1 == ny ? 0u : rw + W) + j);
        const v23 s = ld3(sx, sy, sz, own + pl + rw + j);
        const v23 px = ld3(sx, sy, sz, oth + plp + rw + j);
        const v23 mx = ld3(sx, sy, sz, oth + plm + rw + j);
        const uint32_t p = (x + y + (uint32_t)colour) & 1u;
        const uint32_t je = p ? (j + 2 == W ? 0u : j + 2) : (j == 0 ? W - 1 : j - 1);
        const uint32_t oe = oth + pl + rw + je;
        const float ex = sx[oe], ey = sy[oe], ez = sz[oe];
        pair_compute<MOVE, DMI, HAS_K>(G, rk, status, sx, sy, sz, own + pl + rw + j, x * ny + y, j, p, s, px, mx,
                                       next, prev, cur, ex, ey, ez, sweep, rep, beta2, de, dmx, dmy, dmz);
        prev = cur;
        cur = next;
    }
}

}  // namespace isg
