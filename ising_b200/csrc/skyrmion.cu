// skyrmion.cu -- skyrmion counting on the interpolated winding density:
// calculate_winding_density_interpolated (rsp:366-436), Gaussian_filter_2d (rsp:814-859),
// calculate_skyrmion_number with add_neighbors_to_stack (rsp:582-812) and
// compute_skyrmion_distribution (rsp:930-983), as called by chainMesh_statistics
// (src/PT-Utils.f90:33-66).
//
// Device (FP64): the spins of the first atom of every cell of one slice; their band-limited
// periodic interpolation onto the (sclx*nx) x (scly*ny) fine grid as two matrix products with
// the 1-D interpolation kernels; the fine-grid density; one Gaussian-filtered copy per sigma
// with its largest |value|; per sigma the cells that pass the local-maximum test.
//
// Host: the region growth and merge of calculate_skyrmion_number.  They visit cells in the
// reference's order (a LIFO stack, neighbours -1..1 x -1..1), so each (threshold, sigma) pair
// is sequential; pairs run on all host threads.  The reference wraps every neighbour index
// with the COARSE cell counts (rsp:600-607,713-714,776-777): a fine cell outside the first
// nx x ny block takes part only as a starting cell, and growth touches at most nx*ny cells
// plus the starting cells.  The filter and the window of the first nx x ny cells are all the
// host needs, which replaces the reference's per-call interpolation, full-grid stack clears
// and per-region array resets.
//
// Interpolation: spectral_interpolate_to_fine (rsp:12-70) pads the spectrum of the slice
// with zeros, but its FFTW plans (src/fft.f90:80-84,128-155) take the padded row length
// 2(nx/2+1) as the transform length and write rows of nx/2+2 bins at a pitch of nx/2+1, so
// the values it produces are not reproducible.  This file computes the operation it names:
// the band-limited interpolant through the coarse samples, an even axis's Nyquist term split
// between +n/2 and -n/2.  Every step after the interpolation follows the reference exactly.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "internal.h"
#include "winding.cuh"

namespace isg {
namespace {

#define SKY_TRY(expr)                      \
    do {                                   \
        int st_ = (expr);                  \
        if (st_ != ISING_OK) return st_;   \
    } while (0)

constexpr int kSigmas = 20;            // sigma_index = 1..20 (rsp:962)
constexpr int kStackRows = 10000;      // stack_len (rsp:641)
constexpr double kSkThreshold = 0.05;  // skThreshold (rsp:655)

struct SkyWork {
    int nx = 0, ny = 0, fx = 0, fy = 0, n_sigma = 0;
    double* d_kx = nullptr;     // [nx][fx]: fine row I from coarse row i
    double* d_ky = nullptr;     // [ny][fy]
    double* d_f = nullptr;      // [3][ny][nx]  slice spins, x fastest
    double* d_t = nullptr;      // [3][ny][fx]  after the x pass
    double* d_g = nullptr;      // [3][fy][fx]  fine spins
    double* d_dens = nullptr;   // [fy][fx]     fine density (column-major, x fastest)
    double* d_filt = nullptr;   // [n_sigma][fy][fx]
    double* d_gk = nullptr;     // [n_sigma][25] filter kernels
    unsigned long long* d_max = nullptr;  // [n_sigma] bits of max |filtered|
    int* d_cnt = nullptr;       // [n_sigma] local-maximum cells found
    long long* d_cp = nullptr;  // [n_sigma][fx*fy] their fine index (i-1)*fy + (j-1)
    double* d_cv = nullptr;     // [n_sigma][fx*fy] their filtered value
};

void free_work(SkyWork* w) {
    cudaFree(w->d_kx); cudaFree(w->d_ky); cudaFree(w->d_f); cudaFree(w->d_t); cudaFree(w->d_g);
    cudaFree(w->d_dens); cudaFree(w->d_filt); cudaFree(w->d_gk); cudaFree(w->d_max);
    cudaFree(w->d_cnt); cudaFree(w->d_cp); cudaFree(w->d_cv);
    *w = SkyWork{};
}

template <typename T>
int alloc(T** p, size_t n) {
    cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(ISING_ERR_ALLOC, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    return ISING_OK;
}

// 1-D periodic interpolation kernel from n samples onto M = s*n points, row i of the result
// holding the weights of sample i for fine points I = 0..M-1:
// (1/n) * (1 + 2 sum_{k=1}^{n/2} c_k cos(2 pi k (I - s*i) / M)), c_{n/2} = 1/2 for even n.
std::vector<double> interp_kernel(int n, int s) {
    const int M = n * s, K = n / 2;
    std::vector<double> table(M);
    const double two_pi = 6.283185307179586476925286766559;
    for (int q = 0; q < M; ++q) table[q] = std::cos(two_pi * (double)q / (double)M);
    std::vector<double> k((size_t)n * M);
    for (int i = 0; i < n; ++i)
        for (int I = 0; I < M; ++I) {
            const int64_t d = (int64_t)I - (int64_t)s * i;
            double acc = 0.0;
            for (int f = 1; f <= K; ++f) {
                const int64_t ph = ((f * d) % M + M) % M;
                const double c = (n % 2 == 0 && f == K) ? 0.5 : 1.0;
                acc += c * table[ph];
            }
            k[(size_t)i * M + I] = (1.0 + 2.0 * acc) / (double)n;
        }
    return k;
}

// Gaussian_filter_2d's normalised kernel G(l,m) for l,m = 1..5 (rsp:826-833), row-major.
void gauss_kernel(double sigma, double* G) {
    const int k = 2;
    double acc = 0.0;
    for (int i = 1; i <= 2 * k + 1; ++i)
        for (int j = 1; j <= 2 * k + 1; ++j) {
            const int num = (i - k - 1) * (i - k - 1) + (j - k - 1) * (j - k - 1);
            const double g = std::exp((double)(-num) / (2.0 * (sigma * sigma)));
            G[(i - 1) * 5 + (j - 1)] = g;
            acc = acc + g;
        }
    for (int q = 0; q < 25; ++q) G[q] = G[q] / acc;
}

// sigma of sigma_index si (rsp:964)
double sigma_of(int si) { return 1.0 - ((double)si / 20.0) * (1.0 - 0.00001); }

// ------------------------------------------------------------------ kernels
// map_spins_to_std_grid (src/chainMesh.f90:54-83): spin of the cell's linked-list head
__global__ void k_sky_std_grid(const float* spins, int64_t N, Layout L, int nx, int ny, int z, int sub,
                               double* f) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nx * ny) return;
    const int i = q % nx, j = q / nx;
    const int64_t a = sidx(L, i, j, z, sub);
    const int64_t plane = (int64_t)nx * ny;
    for (int c = 0; c < 3; ++c) f[c * plane + q] = (double)spins[c * N + a];
}

// t[c][j][I] = sum_i kx[i][I] f[c][j][i]
__global__ void k_sky_interp_x(const double* __restrict__ kx, const double* __restrict__ f, int nx, int ny,
                               int fx, double* __restrict__ t) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, c = blockIdx.z;
    if (I >= fx) return;
    const double* row = f + ((int64_t)c * ny + j) * nx;
    double acc = 0.0;
    for (int i = 0; i < nx; ++i) acc = fma(kx[(int64_t)i * fx + I], row[i], acc);
    t[((int64_t)c * ny + j) * fx + I] = acc;
}

// g[c][J][I] = sum_j ky[j][J] t[c][j][I]
__global__ void k_sky_interp_y(const double* __restrict__ ky, const double* __restrict__ t, int ny, int fx,
                               int fy, double* __restrict__ g) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    const int J = blockIdx.y, c = blockIdx.z;
    if (I >= fx) return;
    const double* col = t + (int64_t)c * ny * fx + I;
    double acc = 0.0;
    for (int j = 0; j < ny; ++j) acc = fma(ky[(int64_t)j * fy + J], col[(int64_t)j * fx], acc);
    g[((int64_t)c * fy + J) * fx + I] = acc;
}

__device__ __forceinline__ void unit_at(const double* g, int64_t plane, int64_t q, double* o) {
    const double x = g[q], y = g[plane + q], z = g[2 * plane + q];
    const double n = sqrt(x * x + y * y + z * z);
    o[0] = x / n; o[1] = y / n; o[2] = z / n;
}

// the density loop of calculate_winding_density_interpolated (rsp:409-434)
__global__ void k_sky_density(const double* __restrict__ g, int fx, int fy, double* __restrict__ dens) {
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t plane = (int64_t)fx * fy;
    if (q >= plane) return;
    const int I = (int)(q % fx), J = (int)(q / fx);
    const int I1 = I + 1 == fx ? 0 : I + 1, J1 = J + 1 == fy ? 0 : J + 1;
    double s1[3], s2[3], s3[3], s4[3];
    unit_at(g, plane, q, s1);
    unit_at(g, plane, (int64_t)J * fx + I1, s2);
    unit_at(g, plane, (int64_t)J1 * fx + I1, s3);
    unit_at(g, plane, (int64_t)J1 * fx + I, s4);
    const double w = arc_winding_t<double>(s1, s2, s3) + arc_winding_t<double>(s1, s3, s4);
    dens[q] = w / (4.0 * (double)3.14159265358979323846f);
}

// Gaussian_filter_2d (rsp:836-857) for sigma blockIdx.y: buffer(i,j) = sum_{l,m} array(i-l, j-m)
// G(l,m), l outer, m inner, products and sums rounded separately; then max |value| per sigma.
__global__ void __launch_bounds__(256) k_sky_gauss(const double* __restrict__ a, const double* __restrict__ gk,
                                                   int fx, int fy, double* __restrict__ out,
                                                   unsigned long long* __restrict__ vmax) {
    const int64_t plane = (int64_t)fx * fy;
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    double av = 0.0;
    if (q < plane) {
        const double* G = gk + 25 * s;
        const int i = (int)(q % fx) + 1, j = (int)(q / fx) + 1;
        double acc = 0.0;
        for (int l = 1; l <= 5; ++l) {
            int ii = i - l;
            if (ii < 1) ii = fx - abs(ii);
            for (int m = 1; m <= 5; ++m) {
                int jj = j - m;
                if (jj < 1) jj = fy - abs(jj);
                acc = __dadd_rn(acc, __dmul_rn(a[(int64_t)(jj - 1) * fx + (ii - 1)], G[(l - 1) * 5 + (m - 1)]));
            }
        }
        out[s * plane + q] = acc;
        av = fabs(acc);
    }
    for (int o = 16; o > 0; o >>= 1) av = fmax(av, __shfl_xor_sync(0xffffffffu, av, o));
    __shared__ double wmax[8];
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = av;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = wmax[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, wmax[w]);
        // non-negative doubles order like their bit patterns
        atomicMax(vmax + s, (unsigned long long)__double_as_longlong(m));
    }
}

// The local-maximum test of calculate_skyrmion_number (rsp:709-719) with its coarse wraps;
// cells that pass and lie above tmin * max |value| are listed (in no particular order).
__global__ void k_sky_localmax(const double* __restrict__ filt, const unsigned long long* __restrict__ vmax,
                               int fx, int fy, int nx, int ny, double tmin, int* __restrict__ cnt,
                               long long* __restrict__ cp, double* __restrict__ cv) {
    const int64_t plane = (int64_t)fx * fy;
    const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (q >= plane) return;
    const double* d = filt + s * plane;
    const int I = (int)(q % fx), J = (int)(q / fx);
    const double v = d[q], av = fabs(v);
    bool is_max = true;
    for (int di = -1; di <= 1; ++di)
        for (int dj = -1; dj <= 1; ++dj) {
            if (di == 0 && dj == 0) continue;
            const int x = ((I + di) % nx + nx) % nx, y = ((J + dj) % ny + ny) % ny;
            if (av < fabs(d[(int64_t)y * fx + x])) is_max = false;
        }
    const double mx = __longlong_as_double((long long)vmax[s]);
    if (is_max && av > tmin * mx) {
        const int k = atomicAdd(cnt + s, 1);
        cp[s * plane + k] = (long long)I * fy + J;
        cv[s * plane + k] = v;
    }
}

// ------------------------------------------------------------------ host side
// Runs fn(k, t) for k in [a, b) on up to hardware_concurrency threads, t the thread's index
// (0 .. threads-1), k interleaved over the threads.
int host_threads() { return (int)std::max(1u, std::thread::hardware_concurrency()); }

template <typename Fn>
void parallel_for(int a, int b, const Fn& fn) {
    const int n = b - a;
    const int nt = std::max(1, std::min(n, host_threads()));
    std::vector<std::thread> pool;
    auto work = [&](int t) {
        for (int k = a + t; k < b; k += nt) fn(k, t);
    };
    for (int t = 1; t < nt; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
}

// A cell that passed the local-maximum test: 0-based fine coordinates, its coordinates
// wrapped with the coarse counts (the reference's modulo(i+di-1, nx)+1 before adding di), and
// its filtered value.  Sorted by the reference's loop order, i outer and j inner.
struct Cand {
    int I, J, xm, ym;
    double v;
};

struct SigmaData {
    double max = 0.0;
    std::vector<Cand> c;
    std::vector<double> win;     // filtered values of the first nx x ny cells, x fastest
};

struct Grid {
    int nx, ny, fx, fy;
};

// Region growth (rsp:694-765) for one (threshold, sigma): per region its charge sum, per
// window cell its region, and the starting cells outside the window with their region.  The
// vectors are kept between calls of one host thread.  Returns ISING_ERR_CAPACITY without
// setting the error message (it runs on worker threads).
struct Regions {
    std::vector<double> accs;
    std::vector<int> region;                        // nx*ny, 0 = none
    std::vector<std::pair<int, int>> outside;       // (candidate index, region)
    std::vector<unsigned char> mask, visited, merged;
    std::vector<int> in_stack, stack;
};

int grow_regions(const SigmaData& S, const Grid& g, double thr, Regions* R) {
    const int nx = g.nx, ny = g.ny;
    const size_t nw = (size_t)nx * ny;
    const double cut = thr * S.max;
    R->accs.clear();
    R->outside.clear();
    R->region.assign(nw, 0);
    R->visited.assign(nw, 0);
    R->in_stack.assign(nw, 0);
    R->mask.resize(nw);
    R->stack.resize(kStackRows);
    unsigned char* mask = R->mask.data();
    unsigned char* visited = R->visited.data();
    int* in_stack = R->in_stack.data();
    int* stack = R->stack.data();
    int* region = R->region.data();
    const double* win = S.win.data();
    for (size_t q = 0; q < nw; ++q) mask[q] = std::fabs(win[q]) > cut;
    int rc = 0, sp = 1;
    // one neighbour of add_neighbors_to_stack (rsp:600-616), window index q
    auto consider = [&](int q, double absd) -> bool {
        if (in_stack[q] == rc) return true;
        const bool downhill = absd >= std::fabs(win[q]) - 1e-10;
        if (!visited[q] && mask[q] && downhill) {
            if (sp + 1 > kStackRows) return false;
            stack[sp - 1] = q;
            sp += 1;
            in_stack[q] = rc;
        }
        return true;
    };
    // add_neighbors_to_stack (rsp:582-622) around 0-based fine cell (I, J): indices wrap with the
    // coarse counts (index < 1 -> nx, index > nx -> 1)
    auto push = [&](int I, int J, double absd) -> bool {
        if (I > nx && J > ny) return consider(0, absd);   // all nine map to the window's (1,1)
        for (int di = -1; di <= 1; ++di) {
            int it = I + 1 + di;
            if (it < 1) it = nx;
            if (it > nx) it = 1;
            for (int dj = -1; dj <= 1; ++dj) {
                int jt = J + 1 + dj;
                if (jt < 1) jt = ny;
                if (jt > ny) jt = 1;
                if (!consider((it - 1) + (jt - 1) * nx, absd)) return false;
            }
        }
        return true;
    };
    const int nc = (int)S.c.size();
    for (int k = 0; k < nc; ++k) {
        const Cand& c = S.c[k];
        if (!(std::fabs(c.v) > cut)) continue;
        const bool inwin = c.I < nx && c.J < ny;
        const int qw = inwin ? c.I + c.J * nx : -1;
        if (inwin && visited[qw]) continue;
        R->accs.push_back(c.v);
        rc = (int)R->accs.size();
        if (inwin) {
            visited[qw] = 1;
            region[qw] = rc;
        } else {
            R->outside.emplace_back(k, rc);
        }
        sp = 1;
        if (!push(c.I, c.J, std::fabs(c.v))) return ISING_ERR_CAPACITY;
        while (sp - 1 != 0) {
            const int q = stack[sp - 2];
            sp -= 1;
            if (!visited[q]) {
                R->accs[rc - 1] = R->accs[rc - 1] + win[q];
                visited[q] = 1;
                if (!push(q % nx, q / nx, std::fabs(win[q]))) return ISING_ERR_CAPACITY;
                region[q] = rc;
            }
        }
    }
    return ISING_OK;
}

// The merge loop (rsp:772-805): fine cells with a region in (i, j) order.  A cell of an unmerged
// region whose sum is within 0.05 of particle_number adds sign(sum); otherwise regions whose
// joint sum is within 0.05 are marked merged.
int count_regions(Regions& R, const SigmaData& S, const Grid& g, int particle_number) {
    const int nx = g.nx, ny = g.ny;
    R.merged.assign(R.accs.size(), 0);
    unsigned char* merged = R.merged.data();
    const double* accs = R.accs.data();
    const int* region = R.region.data();
    const double pn = (double)particle_number;
    int sk = 0;
    auto cell = [&](int xm, int ym, int id1) {
        if (merged[id1 - 1]) return;
        const double acc = accs[id1 - 1];
        if (std::fabs(std::fabs(acc) - pn) < kSkThreshold) {
            sk += std::signbit(acc) ? -1 : 1;
            return;
        }
        for (int di = -1; di <= 1; ++di) {
            int x = xm + di;
            if (x < 0) x += nx;
            if (x >= nx) x -= nx;
            for (int dj = -1; dj <= 1; ++dj) {
                if (di == 0 && dj == 0) continue;
                int y = ym + dj;
                if (y < 0) y += ny;
                if (y >= ny) y -= ny;
                const int id2 = region[x + y * nx];
                if (id2 == 0) continue;
                if (merged[id2 - 1]) continue;
                if (std::fabs(std::fabs(accs[id1 - 1] + accs[id2 - 1]) - pn) < kSkThreshold) {
                    merged[id1 - 1] = 1;
                    merged[id2 - 1] = 1;
                }
            }
        }
    };
    size_t o = 0;
    const size_t no = R.outside.size();
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            const long long p = (long long)i * g.fy + j;
            for (; o < no; ++o) {
                const Cand& c = S.c[R.outside[o].first];
                if ((long long)c.I * g.fy + c.J >= p) break;
                cell(c.xm, c.ym, R.outside[o].second);
            }
            const int id = region[i + j * nx];
            if (id) cell(i, j, id);
        }
    for (; o < no; ++o) {
        const Cand& c = S.c[R.outside[o].first];
        cell(c.xm, c.ym, R.outside[o].second);
    }
    return sk;
}

// Device stages on the fine density already in w->d_dens: filters for the given sigmas, max,
// local-maximum lists above tmin * max; downloads everything the host stages read.
int filter_and_collect(SkyWork* w, const std::vector<double>& sigmas, double tmin, cudaStream_t st,
                       std::vector<SigmaData>* out) {
    const int ns = (int)sigmas.size();
    const int64_t plane = (int64_t)w->fx * w->fy;
    std::vector<double> G((size_t)ns * 25);
    for (int s = 0; s < ns; ++s) gauss_kernel(sigmas[s], &G[(size_t)s * 25]);
    ISG_CUDA(cudaMemcpyAsync(w->d_gk, G.data(), G.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    ISG_CUDA(cudaMemsetAsync(w->d_max, 0, ns * sizeof(unsigned long long), st));
    ISG_CUDA(cudaMemsetAsync(w->d_cnt, 0, ns * sizeof(int), st));
    const dim3 grid((unsigned)((plane + 255) / 256), ns);
    k_sky_gauss<<<grid, 256, 0, st>>>(w->d_dens, w->d_gk, w->fx, w->fy, w->d_filt, w->d_max);
    ISG_CUDA(cudaGetLastError());
    k_sky_localmax<<<grid, 256, 0, st>>>(w->d_filt, w->d_max, w->fx, w->fy, w->nx, w->ny, tmin, w->d_cnt, w->d_cp,
                                         w->d_cv);
    ISG_CUDA(cudaGetLastError());
    std::vector<unsigned long long> mx(ns);
    std::vector<int> cnt(ns);
    ISG_CUDA(cudaMemcpyAsync(mx.data(), w->d_max, ns * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    ISG_CUDA(cudaMemcpyAsync(cnt.data(), w->d_cnt, ns * sizeof(int), cudaMemcpyDeviceToHost, st));
    ISG_CUDA(cudaStreamSynchronize(st));
    out->assign(ns, SigmaData{});
    std::vector<std::vector<long long>> cp(ns);
    std::vector<std::vector<double>> cv(ns);
    for (int s = 0; s < ns; ++s) {
        SigmaData& S = (*out)[s];
        double m;
        std::memcpy(&m, &mx[s], sizeof m);
        S.max = m;
        cp[s].resize(cnt[s]);
        cv[s].resize(cnt[s]);
        S.win.resize((size_t)w->nx * w->ny);
        if (cnt[s]) {
            ISG_CUDA(cudaMemcpyAsync(cp[s].data(), w->d_cp + s * plane, cnt[s] * sizeof(long long),
                                     cudaMemcpyDeviceToHost, st));
            ISG_CUDA(cudaMemcpyAsync(cv[s].data(), w->d_cv + s * plane, cnt[s] * sizeof(double),
                                     cudaMemcpyDeviceToHost, st));
        }
        ISG_CUDA(cudaMemcpy2DAsync(S.win.data(), w->nx * sizeof(double), w->d_filt + s * plane,
                                   w->fx * sizeof(double), w->nx * sizeof(double), w->ny, cudaMemcpyDeviceToHost, st));
    }
    ISG_CUDA(cudaStreamSynchronize(st));
    const int nx = w->nx, ny = w->ny, fy = w->fy;
    parallel_for(0, ns, [&](int s, int) {
        SigmaData& S = (*out)[s];
        std::vector<size_t> ord(cp[s].size());
        for (size_t k = 0; k < ord.size(); ++k) ord[k] = k;
        std::sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return cp[s][a] < cp[s][b]; });
        S.c.resize(ord.size());
        for (size_t k = 0; k < ord.size(); ++k) {
            const long long p = cp[s][ord[k]];
            const int I = (int)(p / fy), J = (int)(p % fy);
            S.c[k] = Cand{I, J, I % nx, J % ny, cv[s][ord[k]]};
        }
    });
    return ISING_OK;
}

int ensure_work(SkyWork* w, int nx, int ny, int fx, int fy, int n_sigma) {
    if (w->nx == nx && w->ny == ny && w->fx == fx && w->fy == fy && w->n_sigma >= n_sigma) return ISING_OK;
    free_work(w);
    const size_t plane = (size_t)fx * fy;
    SKY_TRY(alloc(&w->d_kx, (size_t)nx * fx));
    SKY_TRY(alloc(&w->d_ky, (size_t)ny * fy));
    SKY_TRY(alloc(&w->d_f, (size_t)3 * nx * ny));
    SKY_TRY(alloc(&w->d_t, (size_t)3 * ny * fx));
    SKY_TRY(alloc(&w->d_g, 3 * plane));
    SKY_TRY(alloc(&w->d_dens, plane));
    SKY_TRY(alloc(&w->d_filt, (size_t)n_sigma * plane));
    SKY_TRY(alloc(&w->d_gk, (size_t)n_sigma * 25));
    SKY_TRY(alloc(&w->d_max, (size_t)n_sigma));
    SKY_TRY(alloc(&w->d_cnt, (size_t)n_sigma));
    SKY_TRY(alloc(&w->d_cp, (size_t)n_sigma * plane));
    SKY_TRY(alloc(&w->d_cv, (size_t)n_sigma * plane));
    w->nx = nx; w->ny = ny; w->fx = fx; w->fy = fy; w->n_sigma = n_sigma;
    std::vector<double> kx = interp_kernel(nx, fx / nx), ky = interp_kernel(ny, fy / ny);
    ISG_CUDA(cudaMemcpy(w->d_kx, kx.data(), kx.size() * sizeof(double), cudaMemcpyHostToDevice));
    ISG_CUDA(cudaMemcpy(w->d_ky, ky.data(), ky.size() * sizeof(double), cudaMemcpyHostToDevice));
    return ISING_OK;
}

struct Dev {
    int prev = -1;
    explicit Dev(int d) {
        cudaGetDevice(&prev);
        if (prev != d) cudaSetDevice(d);
    }
    ~Dev() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

int check_mesh(const ising_mesh* m, int replica, int z1) {
    if (!m) return fail(ISING_ERR_ARG, "mesh is NULL");
    if (m->device < 0) return fail(ISING_ERR_ARG, "mesh was created without a device (device = -1)");
    if (replica < 0 || replica >= m->n_replicas) return fail(ISING_ERR_BOUNDS, "replica index out of range");
    if (z1 < 1 || z1 > m->lat.nz) return fail(ISING_ERR_BOUNDS, "Z_index out of bounds");
    if ((int64_t)m->lat.nx * m->sclx < 5 || (int64_t)m->lat.ny * m->scly < 5)
        return fail(ISING_ERR_ARG, "fine grid below 5 x 5 (Gaussian_filter_2d reads 5 cells back)");
    if ((int64_t)m->lat.ny * m->scly > 65535 || (int64_t)m->lat.nx * m->sclx * m->lat.ny * m->scly > (int64_t)1 << 31)
        return fail(ISING_ERR_ARG, "fine grid too large (y extent above 65535 or more than 2^31 cells)");
    return mesh_settle(m);   // asynchronous spin transfers land first
}

// slice z1 of one replica -> fine density in w->d_dens
int fine_density(ising_mesh* m, int replica, int z1, int n_sigma, SkyWork** out) {
    if (!m->sky) m->sky = new SkyWork();
    SkyWork* w = static_cast<SkyWork*>(m->sky);
    const Lattice& L = m->lat;
    const int fx = L.nx * m->sclx, fy = L.ny * m->scly;
    SKY_TRY(ensure_work(w, L.nx, L.ny, fx, fy, n_sigma));
    cudaStream_t st = m->stream;
    const float* spins = m->d_spins + (int64_t)replica * 3 * L.natoms;
    k_sky_std_grid<<<(L.nx * L.ny + 255) / 256, 256, 0, st>>>(spins, L.natoms, m->layout, L.nx, L.ny, z1 - 1,
                                                              L.nsub - 1, w->d_f);
    ISG_CUDA(cudaGetLastError());
    k_sky_interp_x<<<dim3((fx + 127) / 128, L.ny, 3), 128, 0, st>>>(w->d_kx, w->d_f, L.nx, L.ny, fx, w->d_t);
    ISG_CUDA(cudaGetLastError());
    k_sky_interp_y<<<dim3((fx + 127) / 128, fy, 3), 128, 0, st>>>(w->d_ky, w->d_t, L.ny, fx, fy, w->d_g);
    ISG_CUDA(cudaGetLastError());
    const int64_t plane = (int64_t)fx * fy;
    k_sky_density<<<(unsigned)((plane + 255) / 256), 256, 0, st>>>(w->d_g, fx, fy, w->d_dens);
    ISG_CUDA(cudaGetLastError());
    *out = w;
    return ISING_OK;
}

// compute_skyrmion_distribution's search (rsp:957-981) over prepared sigma data: results are
// taken in the reference's order; pairs are evaluated speculatively in batches on host threads.
int distribution(const std::vector<SigmaData>& S, const Grid& g, double total_charge, int N, double min_t,
                 double max_t, int num_thresholds, int* winding) {
    std::vector<int> closest(N, 0);
    const long nq = std::lround(total_charge);   // nint for |x| below 2^31
    const int n_pairs = num_thresholds * kSigmas;
    const int batch = 4 * host_threads();
    std::vector<std::vector<int>> res(batch, std::vector<int>(N));
    std::vector<int> status(batch);
    std::vector<Regions> scratch(host_threads());
    for (int j = 0; j < N; ++j) winding[j] = 0;
    for (int base = 0; base < n_pairs; base += batch) {
        const int hi = std::min(n_pairs, base + batch);
        parallel_for(base, hi, [&](int k, int t) {
            const int i = k / kSigmas + 1, si = k % kSigmas + 1;
            const double thr = max_t - ((double)i / (double)num_thresholds) * (max_t - min_t);
            if (std::fabs(thr) > 1.0 || thr < 0.0) {   // the q_threshold check of rsp:689
                status[k - base] = ISING_ERR_ARG;
                return;
            }
            Regions& R = scratch[t];
            status[k - base] = grow_regions(S[si - 1], g, thr, &R);
            if (status[k - base] == ISING_OK)
                for (int j = 1; j <= N; ++j) res[k - base][j - 1] = count_regions(R, S[si - 1], g, j);
        });
        for (int k = base; k < hi; ++k) {
            if (status[k - base] == ISING_ERR_ARG) return fail(ISING_ERR_ARG, "q_threshold must be between 0 and 1");
            if (status[k - base] != ISING_OK) return fail(status[k - base], "Stack array capacity exceeded");
            const std::vector<int>& wa = res[k - base];
            double w = 0.0;
            long cur = 0;
            for (int j = 1; j <= N; ++j) {
                winding[j - 1] = wa[j - 1];
                w = w + (double)(j * wa[j - 1]);
                cur = cur + (long)j * closest[j - 1];
            }
            const long nw = w >= 0.0 ? (long)std::floor(w + 0.5) : -(long)std::floor(-w + 0.5);
            if (std::labs(nw - nq) < std::labs(cur - nq)) closest = wa;
            if (std::fabs(w - total_charge) < 0.1) return ISING_OK;
        }
    }
    for (int j = 0; j < N; ++j) winding[j] = closest[j];
    return ISING_OK;
}

}  // namespace

void skyrmion_release(ising_mesh* m) {
    if (!m || !m->sky) return;
    SkyWork* w = static_cast<SkyWork*>(m->sky);
    free_work(w);
    delete w;
    m->sky = nullptr;
}

}  // namespace isg

using namespace isg;

extern "C" int ising_mesh_set_interpolation_scale(ising_mesh* m, int sclx, int scly) {
    if (!m) return fail(ISING_ERR_ARG, "mesh is NULL");
    if (sclx < 2) return fail(ISING_ERR_ARG, "x interpolation scale must be greater than or equal to 2");
    if (scly < 2) return fail(ISING_ERR_ARG, "y interpolation scale must be greater than or equal to 2");
    m->sclx = sclx;
    m->scly = scly;
    return ISING_OK;
}

extern "C" int ising_mesh_interpolation_scale(const ising_mesh* m, int* sclx, int* scly) {
    if (!m || !sclx || !scly) return fail(ISING_ERR_ARG, "NULL argument");
    *sclx = m->sclx;
    *scly = m->scly;
    return ISING_OK;
}

extern "C" int ising_winding_density_interpolated(const ising_mesh* mc, int replica, int z1, double* density) {
    ising_mesh* m = const_cast<ising_mesh*>(mc);
    SKY_TRY(check_mesh(m, replica, z1));
    if (!density) return fail(ISING_ERR_ARG, "density is NULL");
    Dev d(m->device);
    SkyWork* w = nullptr;
    SKY_TRY(fine_density(m, replica, z1, 1, &w));
    ISG_CUDA(cudaMemcpyAsync(density, w->d_dens, (size_t)w->fx * w->fy * sizeof(double), cudaMemcpyDeviceToHost,
                             m->stream));
    ISG_CUDA(cudaStreamSynchronize(m->stream));
    return ISING_OK;
}

extern "C" int ising_skyrmion_number(const ising_mesh* mc, int replica, int z1, double q_threshold,
                                     int particle_number, double sigma, int* skyrmion_number) {
    ising_mesh* m = const_cast<ising_mesh*>(mc);
    SKY_TRY(check_mesh(m, replica, z1));
    if (!skyrmion_number) return fail(ISING_ERR_ARG, "skyrmion_number is NULL");
    if (std::fabs(q_threshold) > 1.0 || q_threshold < 0.0) return fail(ISING_ERR_ARG, "q_threshold must be between 0 and 1");
    Dev d(m->device);
    SkyWork* w = nullptr;
    SKY_TRY(fine_density(m, replica, z1, 1, &w));
    std::vector<SigmaData> S;
    SKY_TRY(filter_and_collect(w, {sigma}, q_threshold, m->stream, &S));
    const Grid g{w->nx, w->ny, w->fx, w->fy};
    Regions R;
    if (grow_regions(S[0], g, q_threshold, &R) != ISING_OK) return fail(ISING_ERR_CAPACITY, "Stack array capacity exceeded");
    *skyrmion_number = count_regions(R, S[0], g, particle_number);
    return ISING_OK;
}

extern "C" int ising_skyrmion_distribution(const ising_mesh* mc, int replica, int N, double min_threshold,
                                           double max_threshold, int num_thresholds, int z1, int* winding_array) {
    ising_mesh* m = const_cast<ising_mesh*>(mc);
    SKY_TRY(check_mesh(m, replica, z1));
    if (!winding_array || N < 1 || num_thresholds < 1) return fail(ISING_ERR_ARG, "bad distribution arguments");
    if (max_threshold < min_threshold) return fail(ISING_ERR_ARG, "max_threshold must be greater than min_threshold");
    double total = 0.0;
    SKY_TRY(ising_winding_number(m, replica, z1, &total));
    Dev d(m->device);
    SkyWork* w = nullptr;
    SKY_TRY(fine_density(m, replica, z1, kSigmas, &w));
    std::vector<double> sig(kSigmas);
    for (int s = 0; s < kSigmas; ++s) sig[s] = sigma_of(s + 1);
    const double tmin = max_threshold - ((double)num_thresholds / (double)num_thresholds) * (max_threshold - min_threshold);
    std::vector<SigmaData> S;
    SKY_TRY(filter_and_collect(w, sig, std::min(tmin, min_threshold), m->stream, &S));
    return distribution(S, Grid{w->nx, w->ny, w->fx, w->fy}, total, N, min_threshold, max_threshold, num_thresholds,
                        winding_array);
}

extern "C" int ising_chain_mesh_statistics(const ising_mesh* m, int replica, int* skyrmion_number_middle,
                                           double* wnd_mid, double* wnd_spread, double mag[3]) {
    if (!m || !skyrmion_number_middle) return fail(ISING_ERR_ARG, "NULL argument");
    SKY_TRY(ising_statistics(m, replica, wnd_mid, wnd_spread, mag));
    int sk = 0;
    SKY_TRY(ising_skyrmion_distribution(m, replica, 1, 1e-5, 0.95, 60, m->lat.nz / 2, &sk));
    *skyrmion_number_middle = sk;
    return ISING_OK;
}

// On caller-supplied host arrays: the filter and the counting stages of
// calculate_skyrmion_number without the interpolation, on the current device.
namespace {
int host_array_stage(const double* density, int fx, int fy, int nx, int ny, const std::vector<double>& sigmas,
                     double tmin, std::vector<SigmaData>* S, double* filtered_out) {
    SkyWork w;
    w.nx = nx; w.ny = ny; w.fx = fx; w.fy = fy; w.n_sigma = (int)sigmas.size();
    const size_t plane = (size_t)fx * fy;
    int st = ISING_OK;
    cudaStream_t s = nullptr;
    auto run = [&]() -> int {
        SKY_TRY(alloc(&w.d_dens, plane));
        SKY_TRY(alloc(&w.d_filt, sigmas.size() * plane));
        SKY_TRY(alloc(&w.d_gk, sigmas.size() * 25));
        SKY_TRY(alloc(&w.d_max, sigmas.size()));
        SKY_TRY(alloc(&w.d_cnt, sigmas.size()));
        SKY_TRY(alloc(&w.d_cp, sigmas.size() * plane));
        SKY_TRY(alloc(&w.d_cv, sigmas.size() * plane));
        ISG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        ISG_CUDA(cudaMemcpyAsync(w.d_dens, density, plane * sizeof(double), cudaMemcpyHostToDevice, s));
        SKY_TRY(filter_and_collect(&w, sigmas, tmin, s, S));
        if (filtered_out) {
            ISG_CUDA(cudaMemcpyAsync(filtered_out, w.d_filt, plane * sizeof(double), cudaMemcpyDeviceToHost, s));
            ISG_CUDA(cudaStreamSynchronize(s));
        }
        return ISING_OK;
    };
    st = run();
    if (s) cudaStreamDestroy(s);
    free_work(&w);
    return st;
}
}  // namespace

extern "C" int ising_gaussian_filter_2d(double* array, int nx, int ny, double sigma) {
    if (!array) return fail(ISING_ERR_ARG, "array is NULL");
    if (nx < 5 || ny < 5) return fail(ISING_ERR_ARG, "array below 5 x 5 (the filter reads 5 cells back)");
    std::vector<SigmaData> S;
    // the local-maximum stage needs a coarse window; the whole array serves
    return host_array_stage(array, nx, ny, nx, ny, {sigma}, 2.0, &S, array);
}

extern "C" int ising_skyrmion_number_density(const double* density, int fx, int fy, int nx, int ny, double q_threshold,
                                             int particle_number, double sigma, int* skyrmion_number) {
    if (!density || !skyrmion_number) return fail(ISING_ERR_ARG, "NULL argument");
    if (fx < 5 || fy < 5) return fail(ISING_ERR_ARG, "fine grid below 5 x 5 (Gaussian_filter_2d reads 5 cells back)");
    if (nx < 1 || ny < 1 || nx > fx || ny > fy) return fail(ISING_ERR_ARG, "coarse counts must lie in [1, fine counts]");
    if ((int64_t)fx * fy > (int64_t)1 << 31) return fail(ISING_ERR_ARG, "fine grid above 2^31 cells");
    if (std::fabs(q_threshold) > 1.0 || q_threshold < 0.0) return fail(ISING_ERR_ARG, "q_threshold must be between 0 and 1");
    std::vector<SigmaData> S;
    SKY_TRY(host_array_stage(density, fx, fy, nx, ny, {sigma}, q_threshold, &S, nullptr));
    const Grid g{nx, ny, fx, fy};
    Regions R;
    if (grow_regions(S[0], g, q_threshold, &R) != ISING_OK) return fail(ISING_ERR_CAPACITY, "Stack array capacity exceeded");
    *skyrmion_number = count_regions(R, S[0], g, particle_number);
    return ISING_OK;
}
