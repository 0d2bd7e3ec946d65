// device.cuh -- device helpers shared by the sm_100a kernels of libisinggpu.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace isg {

// ---------------------------------------------------------------- Philox4x32
// Counter-based generator of Salmon, Moraes, Dror and Shaw, "Parallel random numbers:
// as easy as 1, 2, 3" (SC'11).  Each round: two 32x32->64 products of the even counter
// words with the published multipliers, an S-box style exchange with the odd words and
// the key, and a Weyl increment of the key.
constexpr uint32_t kPhiloxM0 = 0xD2511F53u;
constexpr uint32_t kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u;
constexpr uint32_t kPhiloxW1 = 0xBB67AE85u;

// Stream tags in the top counter word (low 8 bits); the ensemble id fills the rest.
enum : uint32_t { kTagSweep = 0, kTagInit = 1, kTagExchange = 2, kTagPatch = 3 };

template <int ROUNDS = 10>
__host__ __device__ __forceinline__ uint4 philox4x32(uint4 c, uint2 k) {
#pragma unroll
    for (int i = 0; i < ROUNDS; ++i) {
#ifdef __CUDA_ARCH__
        const uint32_t hi0 = __umulhi(kPhiloxM0, c.x), lo0 = kPhiloxM0 * c.x;
        const uint32_t hi1 = __umulhi(kPhiloxM1, c.z), lo1 = kPhiloxM1 * c.z;
#else
        const uint64_t p0 = (uint64_t)kPhiloxM0 * c.x, p1 = (uint64_t)kPhiloxM1 * c.z;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += kPhiloxW0;
        k.y += kPhiloxW1;
    }
    return c;
}

#if defined(__CUDACC__)
// (0,1) uniform with 23 random bits: (2*(x>>9)+1) * 2^-24, formed exactly as
// (1 + m*2^-23) - (1 - 2^-24) (Sterbenz: the subtraction is exact).
__device__ __forceinline__ float u01(uint32_t x) {
    return __uint_as_float((x >> 9) | 0x3f800000u) - 0.99999994f;
}

// Philox4x32-10 with the ten round keys precomputed (philox_round_keys) and taken from the
// kernel parameters: each round is two 32x32->64 products and two three-input XORs, the
// round keys constant-bank operands.  Same values as philox4x32<10>(c, philox_key(seed)).
__device__ __forceinline__ uint4 philox_rk(uint4 c, const uint32_t* rk) {
#pragma unroll
    for (int i = 0; i < 10; ++i) {
        const uint64_t p0 = (uint64_t)kPhiloxM0 * c.x;
        const uint64_t p1 = (uint64_t)kPhiloxM1 * c.z;
        c = make_uint4((uint32_t)(p1 >> 32) ^ c.y ^ rk[2 * i], (uint32_t)p1,
                       (uint32_t)(p0 >> 32) ^ c.w ^ rk[2 * i + 1], (uint32_t)p0);
    }
    return c;
}

#endif  // __CUDACC__
__host__ __device__ __forceinline__ uint2 philox_key(uint64_t seed) {
    return make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
}
// rk[2i], rk[2i+1] = the key of round i: key + i * (W0, W1)
inline void philox_round_keys(uint64_t seed, uint32_t* rk) {
    uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    for (int i = 0; i < 10; ++i) { rk[2 * i] = k0; rk[2 * i + 1] = k1; k0 += kPhiloxW0; k1 += kPhiloxW1; }
}

// ---------------------------------------------------------------- small vector helpers
struct f3 { float x, y, z; };
#if defined(__CUDACC__)
__device__ __forceinline__ f3 mk(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ float dot(f3 a, f3 b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z)); }
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// Hardware approximations (PTX ISA: sin/cos/ex2/lg2/sqrt/rsqrt .approx).  Their error
// (about 2^-21 relative, 2^-20.5 absolute for sin/cos on [-pi, pi]) is below the FP32 spin
// resolution; the proposals stay symmetric because they depend only on fresh uniforms.
__device__ __forceinline__ float ax_sin(float x) { float y; asm("sin.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x)); return y; }
__device__ __forceinline__ float ax_cos(float x) { float y; asm("cos.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x)); return y; }
__device__ __forceinline__ float ax_ex2(float x) { float y; asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x)); return y; }
__device__ __forceinline__ float ax_lg2(float x) { float y; asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x)); return y; }
__device__ __forceinline__ float ax_sqrt(float x) { float y; asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x)); return y; }
__device__ __forceinline__ float ax_rsqrt(float x) { float y; asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x)); return y; }

// Trial spin from uniforms (u0: cos theta, u1: azimuth, u2: ball radius).
// MOVE 0: fresh uniform unit vector (|v| = 1 to the sin/cos accuracy; not renormalised).
// MOVE 1: S' = norm(S + r*cbrt(u2)*v), the ball move of UniformRandomInSphere
// (reference src/energyMin.f90:49-68).
template <int MOVE>
__device__ __forceinline__ f3 propose(f3 s, float u0, float u1, float u2, float r) {
    const float cz = fmaf(2.0f, u0, -1.0f);                       // exact
    const float st = ax_sqrt(fmaf(-cz, cz, 1.0f));
    const float ph = fmaf(6.28318531f, u1, -3.14159265f);          // azimuth in (-pi, pi), as propose2
    f3 v = {st * ax_cos(ph), st * ax_sin(ph), cz};
    if (MOVE == 1) {
        const float rho = r * ax_ex2(0.33333334f * ax_lg2(u2));   // r * cbrt(u2)
        v = {fmaf(rho, v.x, s.x), fmaf(rho, v.y, s.y), fmaf(rho, v.z, s.z)};
        const float rn = ax_rsqrt(dot(v, v));
        v = {v.x * rn, v.y * rn, v.z * rn};
    }
    return v;
}
#endif  // __CUDACC__

// Unsigned 32-bit division by an invariant divisor (Granlund & Montgomery, PLDI'94, round-up
// method): q = (t + ((n - t) >> 1)) >> (l - 1) with t = mulhi(m, n).
struct FastDiv {
    uint32_t d, m;
    int l;
};
inline FastDiv make_div(uint32_t d) {
    FastDiv f;
    f.d = d;
    int l = 0;
    while ((1ull << l) < d) ++l;
    f.l = l;
    f.m = (uint32_t)((((1ull << l) - d) << 32) / d + 1);
    return f;
}
#if defined(__CUDACC__)
__device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv& f) {
    if (f.l == 0) return n;   // d == 1
    const uint32_t t = __umulhi(f.m, n);
    return (t + ((n - t) >> 1)) >> (f.l - 1);
}
#endif  // __CUDACC__

#if defined(__CUDACC__)
// Trial spins for a pair of sites with packed arithmetic; the MUFU approximations stay scalar.
template <int MOVE>
__device__ __forceinline__ void propose2(const float2* s, uint4 ra, uint4 rb, float r, float2* sp) {
    const float2 one = make_float2(1.f, 1.f);
    const float2 u0 = __fadd2_rn(make_float2(__uint_as_float((ra.x >> 9) | 0x3f800000u),
                                             __uint_as_float((rb.x >> 9) | 0x3f800000u)), make_float2(-0.99999994f, -0.99999994f));
    const float2 u1 = __fadd2_rn(make_float2(__uint_as_float((ra.y >> 9) | 0x3f800000u),
                                             __uint_as_float((rb.y >> 9) | 0x3f800000u)), make_float2(-0.99999994f, -0.99999994f));
    const float2 cz = __ffma2_rn(make_float2(2.f, 2.f), u0, make_float2(-1.f, -1.f));
    const float2 q = __ffma2_rn(make_float2(-cz.x, -cz.y), cz, one);
    const float2 ph = __ffma2_rn(make_float2(6.28318531f, 6.28318531f), u1, make_float2(-3.14159265f, -3.14159265f));
    const float2 st = make_float2(ax_sqrt(q.x), ax_sqrt(q.y));
    float2 vx = __fmul2_rn(st, make_float2(ax_cos(ph.x), ax_cos(ph.y)));
    float2 vy = __fmul2_rn(st, make_float2(ax_sin(ph.x), ax_sin(ph.y)));
    float2 vz = cz;
    if (MOVE == 1) {
        const float2 u2 = __fadd2_rn(make_float2(__uint_as_float((ra.z >> 9) | 0x3f800000u),
                                                 __uint_as_float((rb.z >> 9) | 0x3f800000u)), make_float2(-0.99999994f, -0.99999994f));
        const float2 lg = __fmul2_rn(make_float2(ax_lg2(u2.x), ax_lg2(u2.y)), make_float2(0.33333334f, 0.33333334f));
        const float2 rho = __fmul2_rn(make_float2(r, r), make_float2(ax_ex2(lg.x), ax_ex2(lg.y)));
        vx = __ffma2_rn(rho, vx, s[0]);
        vy = __ffma2_rn(rho, vy, s[1]);
        vz = __ffma2_rn(rho, vz, s[2]);
        const float2 n2 = __ffma2_rn(vx, vx, __ffma2_rn(vy, vy, __fmul2_rn(vz, vz)));
        const float2 rn = make_float2(ax_rsqrt(n2.x), ax_rsqrt(n2.y));
        vx = __fmul2_rn(vx, rn);
        vy = __fmul2_rn(vy, rn);
        vz = __fmul2_rn(vz, rn);
    }
    sp[0] = vx; sp[1] = vy; sp[2] = vz;
}

#endif  // __CUDACC__

// ---------------------------------------------------------------- kernel-facing structs
// FP32 Hamiltonian as the kernels consume it.
struct HamDev {
    float J, Jp;      // shell-1 exchange, shell-2 exchange
    float Bz;         // zeeman_factor * B (field along +z)
    float K;          // anisotropy -K (S.e)^2
    float kx, ky, kz; // anisotropy axis
    float D[6][3];    // simple cubic: D vector per bond direction (+x,-x,+y,-y,+z,-z)
};

// One neighbour slot of a sublattice in a general crystal.
struct Slot {
    int8_t dx, dy, dz;   // cell offset (any sign, wraps periodically)
    uint8_t sub;         // neighbour sublattice
    float w;             // exchange weight (J for shell 1, J' for shell 2)
    float Dx, Dy, Dz;    // DMI vector (zero on shell 2)
};

constexpr int kMaxSub = 16;
constexpr int kMaxSlots = 128;

struct StencilDev {
    const Slot* slots;   // n_sub * kMaxSlots, slot s of sublattice i at [i*kMaxSlots + s]
    const int* count;    // per sublattice
    int nsub;
};

// Storage order of a replica's three spin planes.  cb = 0: the reference atom order.
// cb = 1 (simple-cubic meshes with even extents): colour-separated -- the sites with
// (x+y+z)&1 == 0 first, then colour 1; inside a colour, row order (x, y) with the packed
// z index z>>1, so a colour pass reads and writes whole sectors of its own colour.
// cb = 2 (other crystals with even extents whose couplings never join two sites of one
// sublattice at an all-even non-zero cell offset): octant order -- blocks (octant,
// sublattice rank) of q8 = cells/8 sites, octant = (x&1, y&1, z&1), inside a block the
// packed cell ((x>>1, y>>1), z>>1).  A colour class (octant, sublattice group) is then one
// contiguous range (the sublattices of a group have consecutive ranks), and the neighbours
// of consecutive sites through one stencil slot are consecutive as well.
// cb = 3 (two-sublattice crystals whose first shell only joins the two sublattices, the
// reference's BCC cell): sublattice planes -- all sites of sublattice 0 in (x, y, z) order,
// then sublattice 1, so each sublattice is a colour class of the first shell and a row of one
// sublattice reads consecutive z-sites of the other.
struct Layout {
    int cb;
    int nx, ny, nz, nsub;
    int64_t half;             // sites per colour (cb = 1)
    int64_t q8;               // cells per octant (cb = 2)
    uint8_t srank[kMaxSub];   // cb = 2: storage rank of each sublattice
    uint8_t sofr[kMaxSub];    // cb = 2: sublattice of each rank
};

__host__ __device__ __forceinline__ int64_t sidx(const Layout& L, int ix, int iy, int iz, int sub) {
    if (!L.cb) return (((int64_t)ix * L.ny + iy) * L.nz + iz) * L.nsub + sub;
    if (L.cb == 2) {
        const int oct = ((ix & 1) << 2) | ((iy & 1) << 1) | (iz & 1);
        const int64_t packed = ((int64_t)(ix >> 1) * (L.ny >> 1) + (iy >> 1)) * (L.nz >> 1) + (iz >> 1);
        return ((int64_t)oct * L.nsub + L.srank[sub]) * L.q8 + packed;
    }
    if (L.cb == 3) return (((int64_t)sub * L.nx + ix) * L.ny + iy) * L.nz + iz;   // sublattice planes
    const int c = (ix + iy + iz) & 1;
    return c * L.half + ((int64_t)ix * L.ny + iy) * (L.nz >> 1) + (iz >> 1);
}

// storage index of a reference-order atom index
__host__ __device__ __forceinline__ int64_t sidx_atom(const Layout& L, int64_t atom) {
    if (!L.cb) return atom;
    const int sub = (int)(atom % L.nsub);
    const int64_t cell = atom / L.nsub;
    const int iz = (int)(cell % L.nz);
    const int64_t row = cell / L.nz;
    const int iy = (int)(row % L.ny), ix = (int)(row / L.ny);
    return sidx(L, ix, iy, iz, sub);
}

// Per-replica running accumulators: E, Mx, My, Mz.
struct Acc4 { double e, mx, my, mz; };

// Device status word bits.
enum : int { kStatNan = 1, kStatBounds = 2, kStatTimeout = 4 };

#if defined(__CUDACC__)
__device__ __forceinline__ int wrap(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }
__device__ __forceinline__ int wrap_any(int v, int n) { v %= n; return v < 0 ? v + n : v; }

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
#endif  // __CUDACC__

}  // namespace isg
