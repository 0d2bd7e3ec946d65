// patch_move.cu -- the learned Metropolis-Hastings patch move on simple-cubic meshes and the
// generator of its training samples.  No reference counterpart: the reference proposes
// single-spin moves only (Metropolis_mcs, src/energyMin.f90:234-374); the patch energy uses
// its Hamiltonian terms (calculateHeisenbergEnergy, src/energyMin.f90:86-171).
//
// A patch step updates one class of a 2x2x2 colouring of 4^3 blocks (shifted by a common
// offset), so the 8^3 windows of the patches of a class never contain another patch of the
// class.  For each patch: window x -> network -> per-site tangent proposal (mean mu, spread
// sigma) -> s' = exp_s(omega); window x' -> network -> reverse density of omega_rev =
// log_{s'}(s); accept with min(1, exp(-beta dE) q(x|x') / q(x'|x)).  dE counts every bond of
// the patch once (patch-halo bonds whole, patch-patch bonds half from each end) plus the
// Zeeman and anisotropy terms of the patch sites.  The Jacobian |omega|/sin|omega| of the
// exponential map enters both densities.  A per-slot step scale a and a drift weight l shape
// the tangent move, omega ~ N(a l mu, a^2 sigma^2); both are fixed during a step, so the
// forward and reverse densities use the same a and l.
#include "learned.h"

namespace isg {

struct V3 { float x, y, z; };
__device__ __forceinline__ V3 v3(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ float vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 vcross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
__device__ __forceinline__ V3 vaxpy(float a, V3 x, V3 y) { return {a * x.x + y.x, a * x.y + y.y, a * x.z + y.z}; }
__device__ __forceinline__ V3 vscale(float a, V3 x) { return {a * x.x, a * x.y, a * x.z}; }

// tangent frame at s: helper axis z (x when |s_z| >= 0.9), e1 = normalize(a x s), e2 = s x e1
__device__ __forceinline__ void pframe(V3 s, V3& e1, V3& e2) {
    const V3 a = fabsf(s.z) >= 0.9f ? v3(1.f, 0.f, 0.f) : v3(0.f, 0.f, 1.f);
    e1 = vcross(a, s);
    e1 = vscale(rsqrtf(vdot(e1, e1)), e1);
    e2 = vcross(s, e1);
}
// log(|w| / sin|w|)
__device__ __forceinline__ float log_jac(float th) { return th > 1e-3f ? logf(th / sinf(th)) : th * th * (1.f / 6.f); }


template <typename T>
__device__ __forceinline__ T block_sum64(T v, T* sm) {   // 64 threads
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
    __syncthreads();
    const T r = sm[0] + sm[1];
    __syncthreads();
    return r;
}

__device__ __forceinline__ void patch_origin(const PatchStep& P, int64_t w, int& rep, int& ox, int& oy, int& oz) {
    const int t = (int)(w / P.per_slot);
    const int p = (int)(w - (int64_t)t * P.per_slot);
    rep = P.t2r ? P.t2r[t] : t;
    const int nbz = P.nz / 8, nby = P.ny / 8;
    const int bx = p / (nby * nbz), by = (p / nbz) % nby, bz = p % nbz;
    ox = (8 * bx + 4 * (P.colour & 1) + P.offx) % P.nx;
    oy = (8 * by + 4 * ((P.colour >> 1) & 1) + P.offy) % P.ny;
    oz = (8 * bz + 4 * ((P.colour >> 2) & 1) + P.offz) % P.nz;
}

// windows [nb][3][8][8][8] of windows w0 .. w0+nb-1; patch voxels from prop when given
__global__ void k_patch_gather(PatchStep P, int64_t w0, int nb, const float* __restrict__ prop, float* __restrict__ win,
                               __nv_bfloat16* __restrict__ x0) {
    const int64_t n = (int64_t)nb * 512;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(i / 512), v = (int)(i % 512);
        const int a = v / 64, bb = (v / 8) % 8, c = v % 8;
        int rep, ox, oy, oz;
        patch_origin(P, w0 + b, rep, ox, oy, oz);
        float s[3];
        if (prop && a >= 2 && a < 6 && bb >= 2 && bb < 6 && c >= 2 && c < 6) {
            const int site = ((a - 2) * 4 + (bb - 2)) * 4 + (c - 2);
            for (int q = 0; q < 3; ++q) s[q] = prop[((int64_t)b * 64 + site) * 3 + q];
        } else {
            const int x = (ox - 2 + a + P.nx) % P.nx, y = (oy - 2 + bb + P.ny) % P.ny, z = (oz - 2 + c + P.nz) % P.nz;
            const int64_t si = sidx(P.layout, x, y, z, 0);
            const float* base = P.spins + (int64_t)rep * 3 * P.natoms;
            for (int q = 0; q < 3; ++q) s[q] = base[q * P.natoms + si];
        }
        for (int q = 0; q < 3; ++q) win[((int64_t)b * 3 + q) * 512 + v] = s[q];
        if (x0) {   // the network's input row: 3 channels padded to 8, as k_windows_to_rows writes it
            __nv_bfloat162 h[4];
            h[0] = __floats2bfloat162_rn(s[0], s[1]);
            h[1] = __floats2bfloat162_rn(s[2], 0.f);
            h[2] = __floats2bfloat162_rn(0.f, 0.f);
            h[3] = h[2];
            *reinterpret_cast<uint4*>(x0 + i * 8) = *reinterpret_cast<const uint4*>(h);
        }
    }
}

// one block of 64 threads per window: proposal s' per site, log q(x'|x), rejection flag
__global__ void __launch_bounds__(64) k_patch_propose(PatchStep P, int64_t w0, const float* __restrict__ win,
                                                      const float* __restrict__ out, float* __restrict__ prop,
                                                      double* __restrict__ lqf, int* __restrict__ rej) {
    __shared__ double sd[2];
    __shared__ int si[2];
    const int b = blockIdx.x, i = threadIdx.x;
    const int64_t w = w0 + b;
    const int a = i / 16 + 2, bb = (i / 4) % 4 + 2, c = i % 4 + 2;
    const int v = (a * 8 + bb) * 8 + c;
    const V3 s = v3(win[((int64_t)b * 3) * 512 + v], win[((int64_t)b * 3 + 1) * 512 + v], win[((int64_t)b * 3 + 2) * 512 + v]);
    const float* o = out + ((int64_t)b * 64 + i) * 4;
    const float sc_ = P.step_scale ? P.step_scale[(int)(w / P.per_slot)] : 1.f;
    const float ls = fminf(kLogSigMax, fmaxf(kLogSigMin, o[3])) + logf(sc_);
    const float sig = expf(ls);
    V3 e1, e2;
    pframe(s, e1, e2);
    const V3 mu = vscale(sc_ * P.drift, v3(o[0], o[1], o[2]));
    const uint4 r = philox4x32<10>(make_uint4((uint32_t)(w * 64 + i), P.round, 0u, (P.ensemble << 8) | kTagPatch),
                                   philox_key(P.seed));
    const float u1 = 1.f - u01(r.x), u2 = u01(r.y);
    const float rad = sqrtf(-2.f * logf(u1));
    float sn, cs;
    sincospif(2.f * u2, &sn, &cs);
    const float g1 = rad * cs, g2 = rad * sn;
    const float w1 = vdot(mu, e1) + sig * g1, w2 = vdot(mu, e2) + sig * g2;
    const float th = sqrtf(w1 * w1 + w2 * w2);
    int bad = th >= 3.14159265f ? 1 : 0;
    V3 sp = s;
    if (th > 0.f) {
        const V3 d = vaxpy(w1 / th, e1, vscale(w2 / th, e2));
        sp = vaxpy(cosf(th), s, vscale(sinf(th), d));
        sp = vscale(rsqrtf(vdot(sp, sp)), sp);
    }
    float* pp = prop + ((int64_t)b * 64 + i) * 3;
    pp[0] = sp.x; pp[1] = sp.y; pp[2] = sp.z;
    const double lq = (double)(-0.5f * (g1 * g1 + g2 * g2) - 2.f * ls + log_jac(th));
    const double tot = block_sum64(lq, sd);
    const int nbad = block_sum64(bad, si);
    if (i == 0) { lqf[b] = tot; rej[b] = nbad > 0; }
}

// one block of 64 threads per window: reverse density, patch energy change, accept, write
__global__ void __launch_bounds__(64) k_patch_accept(PatchStep P, int64_t w0, const float* __restrict__ win,
                                                     const float* __restrict__ winp, const float* __restrict__ outp,
                                                     const float* __restrict__ prop, const double* __restrict__ lqf,
                                                     const int* __restrict__ rej, double* __restrict__ dE,
                                                     double* __restrict__ dM, int* __restrict__ accepted) {
    __shared__ double sd[2];
    __shared__ int s_acc;
    const int b = blockIdx.x, i = threadIdx.x;
    const int64_t w = w0 + b;
    const int a = i / 16 + 2, bb = (i / 4) % 4 + 2, c = i % 4 + 2;
    auto at = [&](const float* W, int x, int y, int z) {
        const int vv = (x * 8 + y) * 8 + z;
        return v3(W[((int64_t)b * 3) * 512 + vv], W[((int64_t)b * 3 + 1) * 512 + vv], W[((int64_t)b * 3 + 2) * 512 + vv]);
    };
    const V3 s = at(win, a, bb, c);
    const float* pp = prop + ((int64_t)b * 64 + i) * 3;
    const V3 sp = v3(pp[0], pp[1], pp[2]);
    // reverse proposal density, network output at x'
    const float* o = outp + ((int64_t)b * 64 + i) * 4;
    const float sc_ = P.step_scale ? P.step_scale[(int)(w / P.per_slot)] : 1.f;
    const float ls = fminf(kLogSigMax, fmaxf(kLogSigMin, o[3])) + logf(sc_);
    V3 e1, e2;
    pframe(sp, e1, e2);
    // geodesic distance from both the cosine and the sine (the component of s normal to s'):
    // acos of a cosine near 1 would lose most bits of a small angle
    const float cth = fminf(1.f, fmaxf(-1.f, vdot(sp, s)));
    const V3 vv = vaxpy(-cth, sp, s);
    const float nv = sqrtf(vdot(vv, vv));
    const float th = atan2f(nv, cth);
    const float sc = nv > 1e-12f ? th / nv : 0.f;
    const V3 mu = vscale(sc_ * P.drift, v3(o[0], o[1], o[2]));
    const float r1 = sc * vdot(vv, e1) - vdot(mu, e1), r2 = sc * vdot(vv, e2) - vdot(mu, e2);
    const double lq = (double)(-0.5f * (r1 * r1 + r2 * r2) * expf(-2.f * ls) - 2.f * ls + log_jac(th));
    // energy of site i in x' minus in x; neighbours inside the patch count half
    const HamDev& H = P.ham;
    float de = 0.f;
    const int dxs[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const int x = a + dxs[k][0], y = bb + dxs[k][1], z = c + dxs[k][2];
        const bool inner = x >= 2 && x < 6 && y >= 2 && y < 6 && z >= 2 && z < 6;
        const float wgt = inner ? 0.5f : 1.f;
        const V3 n0 = at(win, x, y, z), n1 = at(winp, x, y, z);
        const V3 D = v3(H.D[k][0], H.D[k][1], H.D[k][2]);
        const float e0 = H.J * vdot(s, n0) + vdot(D, vcross(s, n0));
        const float e1b = H.J * vdot(sp, n1) + vdot(D, vcross(sp, n1));
        de += wgt * (e1b - e0);
    }
    de -= H.Bz * (sp.z - s.z);
    if (H.K != 0.f) {
        const V3 ka = v3(H.kx, H.ky, H.kz);
        const float p1 = vdot(sp, ka), p0 = vdot(s, ka);
        de -= H.K * (p1 * p1 - p0 * p0);
    }
    const double lq_rev = block_sum64(lq, sd);
    const double dE_tot = block_sum64((double)de, sd);
    if (i == 0) {
        const int rep = P.t2r ? P.t2r[(int)(w / P.per_slot)] : (int)(w / P.per_slot);
        const double la = -P.beta_rep[rep] * dE_tot + lq_rev - lqf[b];
        const uint4 r = philox4x32<10>(make_uint4((uint32_t)w, P.round, 1u, (P.ensemble << 8) | kTagPatch), philox_key(P.seed));
        const double u = (double)u01(r.x);
        int ok = !rej[b] && la == la && (la >= 0.0 || log(u) < la);
        if (!(dE_tot == dE_tot)) { ok = 0; atomicOr(P.status, kStatNan); }
        s_acc = ok;
    }
    __syncthreads();
    const int ok = s_acc;
    V3 dm = v3(0.f, 0.f, 0.f);
    if (ok) {
        int rep, ox, oy, oz;
        patch_origin(P, w, rep, ox, oy, oz);
        const int x = (ox + a - 2) % P.nx, y = (oy + bb - 2) % P.ny, z = (oz + c - 2) % P.nz;
        const int64_t si = sidx(P.layout, x, y, z, 0);
        float* base = P.spins + (int64_t)rep * 3 * P.natoms;
        base[si] = sp.x; base[P.natoms + si] = sp.y; base[2 * P.natoms + si] = sp.z;
        dm = v3(sp.x - s.x, sp.y - s.y, sp.z - s.z);
    }
    const double mx = block_sum64((double)dm.x, sd), my = block_sum64((double)dm.y, sd), mz = block_sum64((double)dm.z, sd);
    const double j2 = block_sum64((double)vdot(dm, dm), sd);
    if (i == 0) {
        dE[w] = ok ? dE_tot : 0.0;
        dM[4 * w] = mx; dM[4 * w + 1] = my; dM[4 * w + 2] = mz; dM[4 * w + 3] = j2;
        accepted[w] = ok;
    }
}

// per temperature slot: fold the windows' dE, dM into the replica's accumulators
__global__ void k_patch_fold(PatchStep P, int64_t n_windows, const double* __restrict__ dE, const double* __restrict__ dM,
                             const int* __restrict__ accepted, Acc4* __restrict__ acc,
                             unsigned long long* __restrict__ stats, double* __restrict__ jump) {
    __shared__ double sm[5][8];
    __shared__ long long sa[8];
    const int t = blockIdx.x;
    const int64_t b0 = (int64_t)t * P.per_slot;
    double v[5] = {0, 0, 0, 0, 0};
    long long na = 0;
    for (int64_t w = b0 + threadIdx.x; w < b0 + P.per_slot && w < n_windows; w += blockDim.x) {
        v[0] += dE[w]; v[1] += dM[4 * w]; v[2] += dM[4 * w + 1]; v[3] += dM[4 * w + 2]; v[4] += dM[4 * w + 3];
        na += accepted[w];
    }
    for (int q = 0; q < 5; ++q) v[q] = warp_sum(v[q]);
    na = warp_sum(na);
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    if (lane == 0) { for (int q = 0; q < 5; ++q) sm[q][wp] = v[q]; sa[wp] = na; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot[5] = {0, 0, 0, 0, 0};
        long long ta = 0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { for (int q = 0; q < 5; ++q) tot[q] += sm[q][k]; ta += sa[k]; }
        const int rep = P.t2r ? P.t2r[t] : t;
        acc[rep].e += tot[0]; acc[rep].mx += tot[1]; acc[rep].my += tot[2]; acc[rep].mz += tot[3];
        stats[2 * t] += (unsigned long long)P.per_slot;
        stats[2 * t + 1] += (unsigned long long)ta;
        jump[t] += tot[4];
    }
}

// Training samples: block of 64 threads per window; n_local Metropolis sweeps (two parity
// classes) of the 4^3 patch with the halo fixed, at the beta of the window's replica; the
// final patch spins are the targets [nb][64][3].
__global__ void __launch_bounds__(64) k_patch_equilibrate(PatchStep P, int64_t w0, const float* __restrict__ win,
                                                          int n_local, int move, float r, float* __restrict__ tgt) {
    __shared__ float S[3][512];
    const int b = blockIdx.x, i = threadIdx.x;
    for (int q = 0; q < 3; ++q)
        for (int v = i; v < 512; v += 64) S[q][v] = win[((int64_t)b * 3 + q) * 512 + v];
    __syncthreads();
    const int64_t w = w0 + b;
    const int rep = P.t2r ? P.t2r[(int)(w / P.per_slot)] : (int)(w / P.per_slot);
    const float beta = (float)P.beta_rep[rep];
    const int a = i / 16 + 2, bb = (i / 4) % 4 + 2, c = i % 4 + 2;
    const int v = (a * 8 + bb) * 8 + c;
    const int par = (a + bb + c) & 1;
    const HamDev& H = P.ham;
    const int dxs[6] = {64, -64, 8, -8, 1, -1};
    for (int sw = 0; sw < n_local; ++sw) {
        for (int col = 0; col < 2; ++col) {
            if (par == col) {
                V3 h = v3(0.f, 0.f, -H.Bz);
                for (int k = 0; k < 6; ++k) {
                    const V3 n = v3(S[0][v + dxs[k]], S[1][v + dxs[k]], S[2][v + dxs[k]]);
                    const V3 D = v3(H.D[k][0], H.D[k][1], H.D[k][2]);
                    h = vaxpy(H.J, n, h);
                    const V3 x = vcross(n, D);
                    h = v3(h.x + x.x, h.y + x.y, h.z + x.z);
                }
                const V3 s = v3(S[0][v], S[1][v], S[2][v]);
                const uint4 u = philox4x32<10>(make_uint4((uint32_t)(w * 64 + i), (uint32_t)(2 * sw + col), P.round,
                                                          (P.ensemble << 8) | kTagPatch), philox_key(P.seed ^ 0x5A17ull));
                const f3 t = move == 0 ? propose<0>(f3{s.x, s.y, s.z}, u01(u.x), u01(u.y), u01(u.z), r)
                                       : propose<1>(f3{s.x, s.y, s.z}, u01(u.x), u01(u.y), u01(u.z), r);
                const V3 sp = v3(t.x, t.y, t.z);
                float dE = vdot(v3(sp.x - s.x, sp.y - s.y, sp.z - s.z), h);
                if (H.K != 0.f) {
                    const V3 ka = v3(H.kx, H.ky, H.kz);
                    const float p1 = vdot(sp, ka), p0 = vdot(s, ka);
                    dE -= H.K * (p1 * p1 - p0 * p0);
                }
                if (dE <= 0.f || u01(u.w) < expf(-beta * dE)) { S[0][v] = sp.x; S[1][v] = sp.y; S[2][v] = sp.z; }
            }
            __syncthreads();
        }
    }
    for (int q = 0; q < 3; ++q) tgt[((int64_t)b * 64 + i) * 3 + q] = S[q][v];
}

int launch_patch_gather(const PatchStep& P, int64_t w0, int nb, const float* prop, float* win, cudaStream_t s,
                        __nv_bfloat16* x0) {
    const int64_t n = (int64_t)nb * 512;
    k_patch_gather<<<(int)std::min<int64_t>((n + 255) / 256, 148 * 64), 256, 0, s>>>(P, w0, nb, prop, win, x0);
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}
int launch_patch_propose(const PatchStep& P, int64_t w0, int nb, const float* win, const float* out, float* prop,
                         double* lqf, int* rej, cudaStream_t s) {
    k_patch_propose<<<nb, 64, 0, s>>>(P, w0, win, out, prop, lqf, rej);
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}
int launch_patch_accept(const PatchStep& P, int64_t w0, int nb, const float* win, const float* winp, const float* outp,
                        const float* prop, const double* lqf, const int* rej, double* dE, double* dM, int* acc,
                        cudaStream_t s) {
    k_patch_accept<<<nb, 64, 0, s>>>(P, w0, win, winp, outp, prop, lqf, rej, dE, dM, acc);
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}
int launch_patch_fold(const PatchStep& P, int n_slots, int64_t n_windows, const double* dE, const double* dM,
                      const int* accepted, Acc4* acc, unsigned long long* stats, double* jump, cudaStream_t s) {
    k_patch_fold<<<n_slots, 256, 0, s>>>(P, n_windows, dE, dM, accepted, acc, stats, jump);
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}
int launch_patch_equilibrate(const PatchStep& P, int64_t w0, int nb, const float* win, int n_local, int move, float r,
                             float* tgt, cudaStream_t s) {
    k_patch_equilibrate<<<nb, 64, 0, s>>>(P, w0, win, n_local, move, r, tgt);
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}

}  // namespace isg
