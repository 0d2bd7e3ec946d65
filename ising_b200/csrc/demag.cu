// demag.cu -- the demagnetising field of calculate_demagnetisation_field
// (src/reciprocalSpaceProcesses.f90, rsp:76-281) on the device, in FP64.
//
// 1. Cloud-in-cell deposit (interpolate_to_fft_array, rsp:76-126): one grid point per mesh
//    cell at the cell centre; a cell gathers the spins of the atoms of its 27 neighbouring cells
//    with weight prod_i max(1 - |d_i|, 0), d the atom's offset from the centre in Bravais units
//    (minimum image).  The weights depend only on the atom's sublattice and the cell offset, so
//    they are tabulated once per mesh (taps) from the positions makeChainMesh stores, and the
//    deposit is a gather: no atomics, one thread per cell.
// 2. Forward real-to-complex transform of each component with the x index halved
//    (fft_forward_chainMesh, rsp:178-185), as three direct DFT passes (x real-to-complex, then
//    y and z complex) with exact twiddle tables: a mesh has at most a few hundred cells per
//    axis, so O(n) per output bin costs little next to the sweeps it serves.
// 3. H(k) = -(k.M / k^2) k, the k = 0 bin zero and every bin beyond pi/a, pi/b or pi/c in a
//    Cartesian component zero (rsp:225-262), k = 2 pi (wx/N) ar + 2 pi (wy/L) br + 2 pi (wz/M) cr
//    formed with the reference's operation order (no contraction into FMA).
// 4. Backward transform: inverse complex DFTs along z and y, then the real inverse along x
//    from the N/2+1 stored bins (DC and Nyquist bins by their real parts); the k-space field is
//    not Hermitian in the Nyquist planes of y and z (the folded wave index stays +L/2), and this
//    order fixes what the real inverse means there.  Division by N L M (rsp:266-268).
// 5. The same weights carry the grid field back to the atoms (interpolate_fft_to_atoms,
//    rsp:128-176).
#include <cmath>
#include <memory>
#include <vector>

#include "internal.h"

namespace isg {

namespace {

struct CicTap {
    int8_t dx, dy, dz;   // cell offset of the atom from the cell whose centre gathers it
    uint8_t sub;
    int pad;
    double w;
};

// the reference's pi: a default-real literal (src/constants.f90), pi rounded to single
constexpr double kPiF = (double)3.14159265358979323846f;
// 2 pi in double for the twiddle tables
constexpr double kTwoPi = 6.283185307179586476925286766559;

__device__ __forceinline__ int wrapi(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

// grid[q][c] (c = (iz * ny + iy) * nx + ix) = sum over taps of w * S(cell c + o, sub)
__global__ void k_demag_deposit(const float* spins, int64_t N, Layout L, const CicTap* taps, int ntaps,
                                int nx, int ny, int nz, double* grid) {
    const int64_t ncell = (int64_t)nx * ny * nz;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncell; c += (int64_t)gridDim.x * blockDim.x) {
        const int ix = (int)(c % nx);
        const int64_t r = c / nx;
        const int iy = (int)(r % ny), iz = (int)(r / ny);
        double gx = 0.0, gy = 0.0, gz = 0.0;
        for (int t = 0; t < ntaps; ++t) {
            const CicTap tp = taps[t];
            const int64_t si = sidx(L, wrapi(ix + tp.dx, nx), wrapi(iy + tp.dy, ny), wrapi(iz + tp.dz, nz), tp.sub);
            gx += tp.w * (double)spins[si];
            gy += tp.w * (double)spins[N + si];
            gz += tp.w * (double)spins[2 * N + si];
        }
        grid[c] = gx;
        grid[ncell + c] = gy;
        grid[2 * ncell + c] = gz;
    }
}

// X[q][k][j][i] = sum_n grid[q][k][j][n] e^{-2 pi i i n / nx}, i < nxh
__global__ void k_dft_r2c_x(const double* grid, int nx, int ny, int nz, int nxh, const double2* tw, double2* X) {
    const int64_t nout = 3LL * nz * ny * nxh;
    for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < nout; o += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(o % nxh);
        const int64_t row = o / nxh;   // q, k, j
        const double* g = grid + row * nx;
        double re = 0.0, im = 0.0;
        int m = 0;
        for (int n = 0; n < nx; ++n) {
            re = fma(g[n], tw[m].x, re);
            im = fma(g[n], tw[m].y, im);
            m += i;
            if (m >= nx) m -= nx;
        }
        X[o] = make_double2(re, im);
    }
}

// complex DFT along one axis of [3][nz][ny][nxh] (axis 1: y, stride nxh; axis 2: z, stride
// ny * nxh); sign -1 forward (twiddles as tabulated), +1 inverse (conjugated)
__global__ void k_dft_c2c(const double2* in, double2* out, int nz, int ny, int nxh, int axis, int sign,
                          const double2* tw) {
    const int len = axis == 1 ? ny : nz;
    const int64_t stride = axis == 1 ? nxh : (int64_t)ny * nxh;
    const int64_t total = 3LL * nz * ny * nxh;
    for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < total; o += (int64_t)gridDim.x * blockDim.x) {
        const int64_t rest = o % (stride * len);
        const int kk = (int)(rest / stride);
        const int64_t base = o - (int64_t)kk * stride;
        double re = 0.0, im = 0.0;
        int m = 0;
        for (int n = 0; n < len; ++n) {
            const double2 v = in[base + (int64_t)n * stride];
            const double c = tw[m].x, s = sign < 0 ? tw[m].y : -tw[m].y;
            re = fma(v.x, c, fma(-v.y, s, re));
            im = fma(v.x, s, fma(v.y, c, im));
            m += kk;
            if (m >= len) m -= len;
        }
        out[o] = make_double2(re, im);
    }
}

// H(k) = -(k.M / k^2) k with the cut-off and k = 0 set to zero
__global__ void k_demag_kspace(double2* X, int nx, int ny, int nz, int nxh, const double* kv /* ar, br, cr */,
                               double ca, double cb, double cc) {
    const int64_t nb = (int64_t)nz * ny * nxh;
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < nb; b += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(b % nxh);
        const int64_t r = b / nxh;
        const int j = (int)(r % ny), k = (int)(r / ny);
        const int wx = i;
        const int wy = j > ny / 2 ? j - ny : j;
        const int wz = k > nz / 2 ? k - nz : k;
        // kx = 2*pi*(wx/N)*ar etc., summed kx + ky + kz, without contraction
        const double fx = __dmul_rn(2.0 * kPiF, __ddiv_rn((double)wx, (double)nx));
        const double fy = __dmul_rn(2.0 * kPiF, __ddiv_rn((double)wy, (double)ny));
        const double fz = __dmul_rn(2.0 * kPiF, __ddiv_rn((double)wz, (double)nz));
        double kk[3];
#pragma unroll
        for (int d = 0; d < 3; ++d)
            kk[d] = __dadd_rn(__dadd_rn(__dmul_rn(fx, kv[d]), __dmul_rn(fy, kv[3 + d])), __dmul_rn(fz, kv[6 + d]));
        const double k2 = __dadd_rn(__dadd_rn(__dmul_rn(kk[0], kk[0]), __dmul_rn(kk[1], kk[1])), __dmul_rn(kk[2], kk[2]));
        const int64_t s3 = nb;
        const double2 mx = X[b], my = X[s3 + b], mz = X[2 * s3 + b];
        const bool cut = fabs(kk[0]) > ca || fabs(kk[1]) > cb || fabs(kk[2]) > cc;
        if (b == 0 || cut) {
            X[b] = X[s3 + b] = X[2 * s3 + b] = make_double2(0.0, 0.0);
            continue;
        }
        const double dr = kk[0] * mx.x + kk[1] * my.x + kk[2] * mz.x;
        const double di = kk[0] * mx.y + kk[1] * my.y + kk[2] * mz.y;
        const double qr = -dr / k2, qi = -di / k2;
        X[b] = make_double2(qr * kk[0], qi * kk[0]);
        X[s3 + b] = make_double2(qr * kk[1], qi * kk[1]);
        X[2 * s3 + b] = make_double2(qr * kk[2], qi * kk[2]);
    }
}

// grid[q][k][j][n] = sum_{i < nxh} c_i Re(X[q][k][j][i] e^{+2 pi i i n / nx}) (unnormalised)
__global__ void k_dft_c2r_x(const double2* X, int nx, int ny, int nz, int nxh, const double2* tw, double* grid) {
    const int64_t nout = 3LL * nz * ny * nx;
    for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < nout; o += (int64_t)gridDim.x * blockDim.x) {
        const int n = (int)(o % nx);
        const int64_t row = o / nx;
        const double2* x = X + row * nxh;
        double acc = x[0].x;
        int m = n;
        for (int i = 1; i < nxh; ++i) {
            const bool nyq = (nx % 2 == 0) && i == nx / 2;
            // Re(X e^{+i theta}) = X.re cos theta - X.im sin theta, with tw = e^{-i theta}
            const double v = nyq ? x[i].x * tw[m].x : fma(x[i].x, tw[m].x, x[i].y * tw[m].y);
            acc = nyq ? acc + v : fma(2.0, v, acc);
            m += n;
            if (m >= nx) m -= nx;
        }
        grid[o] = acc;
    }
}

// H of every atom (reference order a = cell * nsub + sub, cell = (ix * ny + iy) * nz + iz):
// sum over the sublattice's taps of w * grid[cell - o] * scale; FP64 reference-order output
// and/or FP32 storage-order planes
__global__ void k_demag_gather(const double* grid, int64_t N, int nsub, int nx, int ny, int nz, const CicTap* taps,
                               const int* tap_start, double scale, Layout L, double* H64, float* H32) {
    const int64_t ncell = (int64_t)nx * ny * nz;
    for (int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; a < N; a += (int64_t)gridDim.x * blockDim.x) {
        const int sub = (int)(a % nsub);
        const int64_t cell = a / nsub;
        const int iz = (int)(cell % nz);
        const int64_t r = cell / nz;
        const int iy = (int)(r % ny), ix = (int)(r / ny);
        double hx = 0.0, hy = 0.0, hz = 0.0;
        for (int t = tap_start[sub]; t < tap_start[sub + 1]; ++t) {
            const CicTap tp = taps[t];
            const int64_t c = ((int64_t)wrapi(iz - tp.dz, nz) * ny + wrapi(iy - tp.dy, ny)) * nx + wrapi(ix - tp.dx, nx);
            hx += tp.w * grid[c];
            hy += tp.w * grid[ncell + c];
            hz += tp.w * grid[2 * ncell + c];
        }
        hx *= scale; hy *= scale; hz *= scale;
        if (H64) { H64[a] = hx; H64[N + a] = hy; H64[2 * N + a] = hz; }
        if (H32) {
            const int64_t si = sidx(L, ix, iy, iz, sub);
            H32[si] = (float)hx; H32[N + si] = (float)hy; H32[2 * N + si] = (float)hz;
        }
    }
}

// per block: sum over its atoms of S . H (FP64), H in reference order
__global__ void k_demag_dot(const float* spins, const double* H64, int64_t N, Layout L, double* partial) {
    __shared__ double red[32];
    double acc = 0.0;
    for (int64_t a = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; a < N; a += (int64_t)gridDim.x * blockDim.x) {
        const int64_t si = sidx_atom(L, a);
        acc += (double)spins[si] * H64[a] + (double)spins[N + si] * H64[N + a] + (double)spins[2 * N + si] * H64[2 * N + a];
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        v = warp_sum(v);
        if (threadIdx.x == 0) partial[blockIdx.x] = v;
    }
}

constexpr int kDotBlocks = 256;

#define DMG_TRY(expr)                    \
    do {                                 \
        int st_ = (expr);                \
        if (st_ != ISING_OK) return st_; \
    } while (0)

template <typename T>
int dalloc(T** p, size_t n) {
    *p = nullptr;
    cudaError_t e = cudaMalloc((void**)p, (n ? n : 1) * sizeof(T));
    if (e != cudaSuccess) return fail(ISING_ERR_ALLOC, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    return ISING_OK;
}

int grid_for(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 148 * 32); }

}  // namespace

struct DemagWork {
    int nx = 0, ny = 0, nz = 0, nxh = 0;
    int64_t ncell = 0;
    int ntaps = 0;
    CicTap* d_taps = nullptr;
    int* d_tap_start = nullptr;
    double* d_grid = nullptr;      // [3][ncell]
    double2* d_a = nullptr;        // [3][nz][ny][nxh]
    double2* d_b = nullptr;
    double2* d_tw[3] = {nullptr, nullptr, nullptr};   // e^{-2 pi i m / n} per axis
    double* d_kv = nullptr;        // ar, br, cr
    double ca = 0, cb = 0, cc = 0; // pi / a, pi / b, pi / c
    double* d_H64 = nullptr;       // [3][natoms] reference order
    float* d_H32 = nullptr;        // [3][natoms] storage order
    double* d_part = nullptr;      // kDotBlocks
};

void demag_release(ising_mesh* m) {
    auto* w = static_cast<DemagWork*>(m->demag);
    if (!w) return;
    cudaFree(w->d_taps); cudaFree(w->d_tap_start); cudaFree(w->d_grid); cudaFree(w->d_a); cudaFree(w->d_b);
    for (auto* t : w->d_tw) cudaFree(t);
    cudaFree(w->d_kv); cudaFree(w->d_H64); cudaFree(w->d_H32); cudaFree(w->d_part);
    delete w;
    m->demag = nullptr;
}

namespace {

int demag_setup(ising_mesh* m, DemagWork** out) {
    if (m->demag) { *out = static_cast<DemagWork*>(m->demag); return ISING_OK; }
    const Lattice& L = m->lat;
    if (L.nx < 3 || L.ny < 3 || L.nz < 3) return fail(ISING_ERR_ARG, "demagnetising field needs 3+ cells per axis");
    std::unique_ptr<DemagWork> w(new DemagWork());
    w->nx = L.nx; w->ny = L.ny; w->nz = L.nz; w->nxh = L.nx / 2 + 1;
    w->ncell = (int64_t)L.nx * L.ny * L.nz;
    // taps: the cell (1,1,1) gathers atom (1+o, sub) with the reference's weight
    std::vector<CicTap> taps;
    std::vector<int> start(1, 0);
    const double c0[3] = {L.av[0] * 1.5 + L.bv[0] * 1.5 + L.cv[0] * 1.5, L.av[1] * 1.5 + L.bv[1] * 1.5 + L.cv[1] * 1.5,
                          L.av[2] * 1.5 + L.bv[2] * 1.5 + L.cv[2] * 1.5};
    const int widths[3] = {L.nx, L.ny, L.nz};
    const double* rv[3] = {L.ar, L.br, L.cr};
    for (int s = 0; s < L.nsub; ++s) {
        for (int ox = -1; ox <= 1; ++ox)
            for (int oy = -1; oy <= 1; ++oy)
                for (int oz = -1; oz <= 1; ++oz) {
                    float p[3];
                    L.position(L.atom_of(1 + ox, 1 + oy, 1 + oz, s), p);
                    const double d[3] = {(double)p[0] - c0[0], (double)p[1] - c0[1], (double)p[2] - c0[2]};
                    double wgt = 1.0;
                    for (int k = 0; k < 3; ++k) {
                        double cf = d[0] * rv[k][0] + d[1] * rv[k][1] + d[2] * rv[k][2];
                        cf -= widths[k] * std::nearbyint(cf / widths[k]);
                        wgt *= std::max(1.0 - std::fabs(cf), 0.0);
                    }
                    if (wgt != 0.0) taps.push_back(CicTap{(int8_t)ox, (int8_t)oy, (int8_t)oz, (uint8_t)s, 0, wgt});
                }
        start.push_back((int)taps.size());
    }
    w->ntaps = (int)taps.size();
    const int64_t nspec = 3LL * L.nz * L.ny * w->nxh;
    int st = ISING_OK;
    auto bail = [&](int code) { m->demag = w.release(); demag_release(m); return code; };
    if ((st = dalloc(&w->d_taps, std::max<size_t>(taps.size(), 1))) || (st = dalloc(&w->d_tap_start, start.size())) ||
        (st = dalloc(&w->d_grid, 3 * (size_t)w->ncell)) || (st = dalloc(&w->d_a, (size_t)nspec)) ||
        (st = dalloc(&w->d_b, (size_t)nspec)) || (st = dalloc(&w->d_kv, 9)) ||
        (st = dalloc(&w->d_H64, 3 * (size_t)L.natoms)) || (st = dalloc(&w->d_H32, 3 * (size_t)L.natoms)) ||
        (st = dalloc(&w->d_part, kDotBlocks)))
        return bail(st);
    for (int k = 0; k < 3; ++k) {
        const int n = widths[k];
        std::vector<double2> tw(n);
        for (int q = 0; q < n; ++q) {
            const double th = kTwoPi * (double)q / (double)n;
            tw[q] = make_double2(std::cos(th), -std::sin(th));
        }
        if ((st = dalloc(&w->d_tw[k], (size_t)n)) != ISING_OK) return bail(st);
        if (cudaMemcpy(w->d_tw[k], tw.data(), n * sizeof(double2), cudaMemcpyHostToDevice) != cudaSuccess)
            return bail(cuda_fail(cudaGetLastError(), "demag twiddles"));
    }
    const double kv[9] = {L.ar[0], L.ar[1], L.ar[2], L.br[0], L.br[1], L.br[2], L.cr[0], L.cr[1], L.cr[2]};
    if (cudaMemcpy(w->d_kv, kv, sizeof kv, cudaMemcpyHostToDevice) != cudaSuccess ||
        (!taps.empty() && cudaMemcpy(w->d_taps, taps.data(), taps.size() * sizeof(CicTap), cudaMemcpyHostToDevice) != cudaSuccess) ||
        cudaMemcpy(w->d_tap_start, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(cuda_fail(cudaGetLastError(), "demag tables"));
    // the cut-off uses the lattice constants a, b, c (chainMesh%a, %b, %c)
    w->ca = kPiF / L.a; w->cb = kPiF / L.b; w->cc = kPiF / L.c;
    m->demag = w.release();
    *out = static_cast<DemagWork*>(m->demag);
    return ISING_OK;
}

}  // namespace

int demag_enqueue(ising_mesh* m, int replica, bool want64, bool want32) {
    DemagWork* w = nullptr;
    DMG_TRY(demag_setup(m, &w));
    const Lattice& L = m->lat;
    const int64_t N = L.natoms;
    const float* spins = m->d_spins + (int64_t)replica * 3 * N;
    cudaStream_t s = m->stream;
    const int nx = w->nx, ny = w->ny, nz = w->nz, nxh = w->nxh;
    const int64_t nspec = 3LL * nz * ny * nxh;
    k_demag_deposit<<<grid_for(w->ncell), 256, 0, s>>>(spins, N, m->layout, w->d_taps, w->ntaps, nx, ny, nz, w->d_grid);
    k_dft_r2c_x<<<grid_for(nspec), 256, 0, s>>>(w->d_grid, nx, ny, nz, nxh, w->d_tw[0], w->d_a);
    k_dft_c2c<<<grid_for(nspec), 256, 0, s>>>(w->d_a, w->d_b, nz, ny, nxh, 1, -1, w->d_tw[1]);
    k_dft_c2c<<<grid_for(nspec), 256, 0, s>>>(w->d_b, w->d_a, nz, ny, nxh, 2, -1, w->d_tw[2]);
    k_demag_kspace<<<grid_for(nspec / 3), 256, 0, s>>>(w->d_a, nx, ny, nz, nxh, w->d_kv, w->ca, w->cb, w->cc);
    k_dft_c2c<<<grid_for(nspec), 256, 0, s>>>(w->d_a, w->d_b, nz, ny, nxh, 2, +1, w->d_tw[2]);
    k_dft_c2c<<<grid_for(nspec), 256, 0, s>>>(w->d_b, w->d_a, nz, ny, nxh, 1, +1, w->d_tw[1]);
    k_dft_c2r_x<<<grid_for(3 * w->ncell), 256, 0, s>>>(w->d_a, nx, ny, nz, nxh, w->d_tw[0], w->d_grid);
    k_demag_gather<<<grid_for(N), 256, 0, s>>>(w->d_grid, N, L.nsub, nx, ny, nz, w->d_taps, w->d_tap_start,
                                               1.0 / (double)w->ncell, m->layout, want64 ? w->d_H64 : nullptr,
                                               want32 ? w->d_H32 : nullptr);
    ISG_CUDA(cudaGetLastError());
    return ISING_OK;
}

const double* demag_field64(const ising_mesh* m) { return m->demag ? static_cast<DemagWork*>(m->demag)->d_H64 : nullptr; }
const float* demag_field32(const ising_mesh* m) { return m->demag ? static_cast<DemagWork*>(m->demag)->d_H32 : nullptr; }

int demag_dot(ising_mesh* m, int replica, double* out) {
    auto* w = static_cast<DemagWork*>(m->demag);
    if (!w) return fail(ISING_ERR_ARG, "demagnetising field not computed");
    const int64_t N = m->lat.natoms;
    k_demag_dot<<<kDotBlocks, 256, 0, m->stream>>>(m->d_spins + (int64_t)replica * 3 * N, w->d_H64, N, m->layout,
                                                   w->d_part);
    ISG_CUDA(cudaGetLastError());
    std::vector<double> h(kDotBlocks);
    ISG_CUDA(cudaMemcpyAsync(h.data(), w->d_part, kDotBlocks * sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    ISG_CUDA(cudaStreamSynchronize(m->stream));
    double t = 0.0;
    for (double v : h) t += v;
    *out = t;
    return ISING_OK;
}

}  // namespace isg
