// lattice.cpp -- host lattice compiler of libisinggpu.
//
// Turns "unit cell + Bravais parameters" into per-sublattice neighbour stencils with the
// semantics of the reference's makeChainMesh (src/chainMesh.f90:729-911): Bravais and dual
// vectors, real(4) atom positions, minimum-image distances, distance shells
// (initAtomShells :495-591), the legacy nearest-neighbour list (assignNearestNeighbors
// :280-405) and the per-axis neighbours (DerivativeList :931-1031).  The reference scans
// 125 cells per atom; the periodic mesh is translation invariant, so here each list is
// built once per sublattice at cell 0 and applied to every cell by offset.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "internal.h"

namespace isg {

namespace {
// the reference's pi is a default-real literal (src/constants.f90:16)
const double kPiF = (double)3.14159265358979323846f;

long f_nint(double x) { return (long)(x >= 0.0 ? std::floor(x + 0.5) : -std::floor(-x + 0.5)); }
int pmod(long a, int n) { long r = a % n; return (int)(r < 0 ? r + n : r); }
void cross3(const double* a, const double* b, double* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

struct Cand {
    int dx, dy, dz, sub;
    float x, y, z;   // real(4) position
};

// Minimum-image Bravais coefficients of q - p from double positions
// (distance_points_vec_bravais, src/chainMesh.f90:244-276).
void coeffs(const Lattice& L, const double p[3], const double q[3], double co[3]) {
    double d[3] = {q[0] - p[0], q[1] - p[1], q[2] - p[2]};
    double ac = d[0] * L.ar[0] + d[1] * L.ar[1] + d[2] * L.ar[2];
    double bc = d[0] * L.br[0] + d[1] * L.br[1] + d[2] * L.br[2];
    double cc = d[0] * L.cr[0] + d[1] * L.cr[1] + d[2] * L.cr[2];
    co[0] = ac - (double)L.nx * (double)f_nint(ac / (double)L.nx);
    co[1] = bc - (double)L.ny * (double)f_nint(bc / (double)L.ny);
    co[2] = cc - (double)L.nz * (double)f_nint(cc / (double)L.nz);
}

// distance_points_vec (:206-241): min-image Cartesian r = q - p
void min_image(const Lattice& L, const double p[3], const double q[3], double r[3]) {
    double co[3];
    coeffs(L, p, q, co);
    for (int k = 0; k < 3; ++k) r[k] = co[0] * L.av[k] + co[1] * L.bv[k] + co[2] * L.cv[k];
}

// distance (:133-169): single-precision coordinate differences, real(4) result
float distance_f(const Lattice& L, const float p[3], const float q[3]) {
    double d[3] = {(double)(q[0] - p[0]), (double)(q[1] - p[1]), (double)(q[2] - p[2])};
    double ac = d[0] * L.ar[0] + d[1] * L.ar[1] + d[2] * L.ar[2];
    double bc = d[0] * L.br[0] + d[1] * L.br[1] + d[2] * L.br[2];
    double cc = d[0] * L.cr[0] + d[1] * L.cr[1] + d[2] * L.cr[2];
    ac -= (double)L.nx * (double)f_nint(ac / (double)L.nx);
    bc -= (double)L.ny * (double)f_nint(bc / (double)L.ny);
    cc -= (double)L.nz * (double)f_nint(cc / (double)L.nz);
    double r[3];
    for (int k = 0; k < 3; ++k) r[k] = ac * L.av[k] + bc * L.bv[k] + cc * L.cv[k];
    return (float)std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
}

// Bottom-up pairwise merge sort that takes the right run's element on ties, matching
// merge_dp (src/algo.f90:353-420) so equal-distance neighbours keep the reference order.
void merge_sort_ref(std::vector<double>& a, std::vector<int>& comp) {
    const int n = (int)a.size();
    if (n <= 1) return;
    std::vector<int> lo(n), hi(n);
    std::vector<double> sa(n);
    std::vector<int> sc(n);
    for (int i = 0; i < n; ++i) lo[i] = hi[i] = i;
    int nb = n;
    while (nb > 1) {
        int cnt = 0;
        for (int i = 0; i < nb / 2; ++i) {
            int a0 = lo[2 * i], a1 = hi[2 * i], b0 = lo[2 * i + 1], b1 = hi[2 * i + 1];
            int ia = a0, ib = b0, k = 0;
            while (ia <= a1 && ib <= b1) {
                if (a[ia] < a[ib]) { sa[k] = a[ia]; sc[k] = comp[ia]; ++ia; }
                else { sa[k] = a[ib]; sc[k] = comp[ib]; ++ib; }
                ++k;
            }
            while (ia <= a1) { sa[k] = a[ia]; sc[k] = comp[ia]; ++ia; ++k; }
            while (ib <= b1) { sa[k] = a[ib]; sc[k] = comp[ib]; ++ib; ++k; }
            std::copy(sa.begin(), sa.begin() + k, a.begin() + a0);
            std::copy(sc.begin(), sc.begin() + k, comp.begin() + a0);
            lo[cnt] = a0; hi[cnt] = b1; ++cnt;
        }
        if (nb % 2) { lo[cnt] = lo[nb - 1]; hi[cnt] = hi[nb - 1]; ++cnt; }
        nb = cnt;
    }
}
}  // namespace

void Lattice::cell_of(int64_t atom, int* ix, int* iy, int* iz, int* sub) const {
    *sub = (int)(atom % nsub);
    int64_t cell = atom / nsub;
    *iz = (int)(cell % nz);
    int64_t r = cell / nz;
    *iy = (int)(r % ny);
    *ix = (int)(r / ny);
}

void Lattice::position(int64_t atom, float out[3]) const {
    int ix, iy, iz, s;
    cell_of(atom, &ix, &iy, &iz, &s);
    double fx = frac[3 * s], fy = frac[3 * s + 1], fz = frac[3 * s + 2];
    for (int k = 0; k < 3; ++k) {
        double t = av[k] * (double)ix + bv[k] * (double)iy + cv[k] * (double)iz;
        double p = fx * av[k] + fy * bv[k] + fz * cv[k];
        out[k] = (float)(p + t);
    }
}

int64_t Lattice::neighbour_atom(int64_t atom, const NbrSlot& s) const {
    int ix, iy, iz, sub;
    cell_of(atom, &ix, &iy, &iz, &sub);
    return atom_of(pmod(ix + s.dx, nx), pmod(iy + s.dy, ny), pmod(iz + s.dz, nz), s.sub);
}

int build_lattice(const float* frac, int nsub, int nx, int ny, int nz, double a, double b,
                  double c, double ab_deg, double bc_deg, double ca_deg, double shell_tol,
                  int n_shells, Lattice* out) {
    if (!frac) return fail(ISING_ERR_ARG, "frac_xyz is NULL");
    if (nsub < 1 || nsub > kMaxSub) return fail(ISING_ERR_ARG, "n_atoms_cell must be in 1..16");
    if (nx < 3 || ny < 3 || nz < 3)
        return fail(ISING_ERR_ARG, "nx, ny, nz must be >= 3 (derivativeList needs distinct neighbour cells)");
    if (!(a > 0 && b > 0 && c > 0)) return fail(ISING_ERR_ARG, "lattice constants must be positive");
    for (int i = 0; i < 3 * nsub; ++i)
        if (!std::isfinite(frac[i])) return fail(ISING_ERR_NAN, "non-finite fractional coordinate");
    Lattice& L = *out;
    L = Lattice();
    L.nx = nx; L.ny = ny; L.nz = nz; L.nsub = nsub;
    L.nshells = n_shells > 0 ? n_shells : 2;
    if (L.nshells > 4) return fail(ISING_ERR_ARG, "n_shells must be <= 4");
    const double thr = shell_tol > 0.0 ? shell_tol : 0.1 * a;
    L.a = a; L.b = b; L.c = c;
    L.ncells = (int64_t)nx * ny * nz;
    L.natoms = L.ncells * nsub;
    if (L.natoms > (int64_t)INT32_MAX) return fail(ISING_ERR_ARG, "more than 2^31-1 atoms");
    L.frac.assign(frac, frac + 3 * nsub);

    // Bravais vectors (:798-815) including the reference's c_y expression (:801) and the
    // 1e-5 clean-up; dual basis (:823-825).
    const double ab = ab_deg * (kPiF / 180.0), bc = bc_deg * (kPiF / 180.0), ca = ca_deg * (kPiF / 180.0);
    L.av[0] = a; L.av[1] = 0.0; L.av[2] = 0.0;
    L.bv[0] = b * std::cos(ab); L.bv[1] = b * std::sin(ab); L.bv[2] = 0.0;
    const double cx = c * std::cos(ca);
    const double cy = (c * b * std::cos(bc) - cx * L.bv[0]);
    const double cz2 = c * c - cx * cx - cy * cy;
    if (!(cz2 > 0.0)) return fail(ISING_ERR_ARG, "cell angles give no c_z component");
    L.cv[0] = cx; L.cv[1] = cy; L.cv[2] = std::sqrt(cz2);
    for (int k = 0; k < 3; ++k) {
        if (!(std::fabs(L.av[k]) > 1e-5)) L.av[k] = 0.0;
        if (!(std::fabs(L.bv[k]) > 1e-5)) L.bv[k] = 0.0;
        if (!(std::fabs(L.cv[k]) > 1e-5)) L.cv[k] = 0.0;
    }
    double t[3];
    cross3(L.bv, L.cv, t); { double s = dot3(L.av, t); for (int k = 0; k < 3; ++k) L.ar[k] = t[k] / s; }
    cross3(L.cv, L.av, t); { double s = dot3(L.bv, t); for (int k = 0; k < 3; ++k) L.br[k] = t[k] / s; }
    cross3(L.av, L.bv, t); { double s = dot3(L.cv, t); for (int k = 0; k < 3; ++k) L.cr[k] = t[k] / s; }

    auto pos_of = [&](int ix, int iy, int iz, int s, float p[3]) {
        L.position(L.atom_of(ix, iy, iz, s), p);
    };
    auto dpos = [](const float p[3], double d[3]) { for (int k = 0; k < 3; ++k) d[k] = (double)p[k]; };

    L.shell[0].assign(nsub, {});
    L.shell[1].assign(nsub, {});
    L.legacy.assign(nsub, {});
    L.deriv.assign((size_t)nsub * 6, NbrSlot{0, 0, 0, 0, {0, 0, 0}});

    const int N = L.nshells;
    for (int i = 0; i < nsub; ++i) {
        float pi[3];
        pos_of(0, 0, 0, i, pi);
        double pid[3];
        dpos(pi, pid);

        // ---- shells: (2N+1)^3 cells in NNearestCells order (:618-634), atoms of each cell in
        // linked-list order (last unit-cell atom first, addAtomToChainCell :663-671)
        std::vector<Cand> cand;
        for (int di = -N; di <= N; ++di)
            for (int dj = -N; dj <= N; ++dj)
                for (int dk = -N; dk <= N; ++dk)
                    for (int s = nsub - 1; s >= 0; --s) {
                        int cx_ = pmod(di, nx), cy_ = pmod(dj, ny), cz_ = pmod(dk, nz);
                        if (cx_ == 0 && cy_ == 0 && cz_ == 0 && s == i) continue;  // itself
                        Cand q{di, dj, dk, s, 0, 0, 0};
                        float p[3];
                        pos_of(cx_, cy_, cz_, s, p);
                        q.x = p[0]; q.y = p[1]; q.z = p[2];
                        cand.push_back(q);
                    }
        const int cap = (2 * N + 1) * (2 * N + 1) * (2 * N + 1) * nsub;
        std::vector<double> dist(cap, 1.7976931348623157e308);
        std::vector<int> idx(cap, -1);
        for (size_t q = 0; q < cand.size(); ++q) {
            float p[3] = {cand[q].x, cand[q].y, cand[q].z};
            dist[q] = (double)distance_f(L, pi, p);
            idx[q] = (int)q;
        }
        merge_sort_ref(dist, idx);
        int shell = 0;
        auto push = [&](int q, int sh) {
            if (sh > 1) return;  // only shells 1 and 2 enter the energies
            const Cand& cd = cand[q];
            NbrSlot ns{cd.dx, cd.dy, cd.dz, cd.sub, {0, 0, 0}};
            float p[3] = {cd.x, cd.y, cd.z};
            double pd[3];
            dpos(p, pd);
            min_image(L, pid, pd, ns.r);
            L.shell[sh][i].push_back(ns);
        };
        if (idx[0] >= 0) push(idx[0], 0);
        for (int q = 1; q < cap; ++q) {
            if (idx[q] < 0) break;
            if (std::fabs(dist[q] - dist[q - 1]) > thr) ++shell;
            if (shell >= N) break;
            push(idx[q], shell);
        }
        if ((int)L.shell[0][i].size() > kMaxSlots || (int)L.shell[1][i].size() > kMaxSlots)
            return fail(ISING_ERR_ARG, "neighbour shell larger than the 128-slot stencil limit");

        // ---- legacy NeighborList: 27 cells (getNeighboringCells :85-131), dedup by atom,
        // |d - d_min| < a/100 in single precision (:299-357)
        std::vector<Cand> c27;
        for (int di = -1; di <= 1; ++di)
            for (int dj = -1; dj <= 1; ++dj)
                for (int dk = -1; dk <= 1; ++dk)
                    for (int s = nsub - 1; s >= 0; --s) {
                        int cx_ = pmod(di, nx), cy_ = pmod(dj, ny), cz_ = pmod(dk, nz);
                        if (cx_ == 0 && cy_ == 0 && cz_ == 0 && s == i) continue;
                        float p[3];
                        pos_of(cx_, cy_, cz_, s, p);
                        c27.push_back(Cand{di, dj, dk, s, p[0], p[1], p[2]});
                    }
        float nnd = 3.4028235e38f;
        for (auto& q : c27) {
            float p[3] = {q.x, q.y, q.z};
            float d = distance_f(L, pi, p);
            if (d < nnd) nnd = d;
        }
        std::vector<int64_t> seen;
        for (auto& q : c27) {
            int64_t at = L.atom_of(pmod(q.dx, nx), pmod(q.dy, ny), pmod(q.dz, nz), q.sub);
            if (std::find(seen.begin(), seen.end(), at) != seen.end()) continue;
            float p[3] = {q.x, q.y, q.z};
            float d = distance_f(L, pi, p);
            if (std::fabs((double)(d - nnd)) < a / 100.0) {
                seen.push_back(at);
                NbrSlot ns{q.dx, q.dy, q.dz, q.sub, {0, 0, 0}};
                double pd[3];
                dpos(p, pd);
                min_image(L, pid, pd, ns.r);
                L.legacy[i].push_back(ns);
            }
        }
        if ((int)L.legacy[i].size() > kMaxSlots)
            return fail(ISING_ERR_ARG, "legacy neighbour list larger than 128 slots");

        // ---- derivative list (:956-1031): other cells only, the two other Bravais
        // coefficients within 1e-4, nearest below / above along d, ties to the later atom
        for (int d = 0; d < 3; ++d) {
            int imin = -1, imax = -1;
            double cmin = 1.7976931348623157e308, cmax = cmin;
            for (size_t q = 0; q < c27.size(); ++q) {
                const Cand& cd = c27[q];
                if (pmod(cd.dx, nx) == 0 && pmod(cd.dy, ny) == 0 && pmod(cd.dz, nz) == 0) continue;
                float p[3] = {cd.x, cd.y, cd.z};
                double pd[3], co[3];
                dpos(p, pd);
                coeffs(L, pid, pd, co);
                bool ok = true;
                for (int j = 0; j < 3; ++j)
                    if (j != d && std::fabs(co[j]) > 0.0001) { ok = false; break; }
                if (!ok) continue;
                if (co[d] < 0.0 && std::fabs(co[d]) <= cmin) { cmin = std::fabs(co[d]); imin = (int)q; }
                if (co[d] > 0.0 && std::fabs(co[d]) <= cmax) { cmax = std::fabs(co[d]); imax = (int)q; }
            }
            if (imin < 0 || imax < 0) { L.deriv_ok = false; continue; }
            const Cand& lo = c27[imin];
            const Cand& hi = c27[imax];
            L.deriv[i * 6 + d * 2 + 0] = NbrSlot{lo.dx, lo.dy, lo.dz, lo.sub, {0, 0, 0}};
            L.deriv[i * 6 + d * 2 + 1] = NbrSlot{hi.dx, hi.dy, hi.dz, hi.sub, {0, 0, 0}};
        }
    }
    if (!L.deriv_ok) return fail(ISING_ERR_LATTICE, "Unable to locate atoms (derivative list incomplete)");
    return ISING_OK;
}

int greedy_colouring(const Lattice& L, bool use_shell2, std::vector<int>* colour, int* ncol) {
    const int64_t n = L.natoms;
    colour->assign((size_t)n, -1);
    int maxc = 0;
    std::vector<char> used(2 * kMaxSlots + 2);
    for (int64_t at = 0; at < n; ++at) {
        int ix, iy, iz, s;
        L.cell_of(at, &ix, &iy, &iz, &s);
        std::fill(used.begin(), used.end(), 0);
        for (int sh = 0; sh < (use_shell2 ? 2 : 1); ++sh)
            for (const NbrSlot& q : L.shell[sh][s]) {
                int64_t j = L.neighbour_atom(at, q);
                int cj = (*colour)[j];
                if (j != at && cj >= 0 && cj < (int)used.size()) used[cj] = 1;
            }
        int cc = 0;
        while (used[cc]) ++cc;
        (*colour)[at] = cc;
        maxc = std::max(maxc, cc + 1);
    }
    // verify: no bond inside a class (either direction)
    for (int64_t at = 0; at < n; ++at) {
        int ix, iy, iz, s;
        L.cell_of(at, &ix, &iy, &iz, &s);
        for (int sh = 0; sh < (use_shell2 ? 2 : 1); ++sh)
            for (const NbrSlot& q : L.shell[sh][s]) {
                int64_t j = L.neighbour_atom(at, q);
                if (j == at) return fail(ISING_ERR_LATTICE, "self bond: mesh too small for the active shells");
                if ((*colour)[j] == (*colour)[at]) return fail(ISING_ERR_LATTICE, "colouring is not an independent set");
            }
    }
    *ncol = maxc;
    return ISING_OK;
}

// Sublattice-plane order (layout 3): two sublattices whose first shell joins each site to
// exactly the 8 sites of the other sublattice in the cells base + {0,1}^3 (the reference's BCC
// cell: base (-1,-1,-1) for the corner atom, (0,0,0) for the body centre).  Each sublattice
// is then a colour class of the first shell.  base[s][axis] receives the offsets.
bool bipartite_pair(const Lattice& L, int base[2][3]) {
    if (L.nsub != 2) return false;
    for (int s = 0; s < 2; ++s) {
        const auto& sh = L.shell[0][s];
        if (sh.size() != 8) return false;
        int lo[3] = {1 << 20, 1 << 20, 1 << 20};
        for (const auto& q : sh) {
            if (q.sub != 1 - s) return false;
            lo[0] = std::min(lo[0], q.dx); lo[1] = std::min(lo[1], q.dy); lo[2] = std::min(lo[2], q.dz);
        }
        int seen = 0;
        for (const auto& q : sh) {
            const int a = q.dx - lo[0], b = q.dy - lo[1], c = q.dz - lo[2];
            if (a < 0 || a > 1 || b < 0 || b > 1 || c < 0 || c > 1) return false;
            seen |= 1 << (a * 4 + b * 2 + c);
        }
        if (seen != 0xff) return false;
        for (int k = 0; k < 3; ++k) {
            if (lo[k] < -1 || lo[k] > 0) return false;
            base[s][k] = lo[k];
        }
    }
    return true;
}

// Octant colouring of a general crystal: class (cell octant (x&1, y&1, z&1), sublattice
// group).  Valid when every extent is even (periodic wraps keep parities) and no bond of
// shells 1-2 joins two sites of one sublattice at an all-even non-zero cell offset; two
// sublattices joined by a bond at an all-even offset (including 0) go to different groups
// (greedy colouring of that small graph).  A bond of a site to itself, which the reference's
// shell search puts into shell 2 of BCC cells, does not constrain the colouring: the update
// reads the site's own old value there, as a sequential sweep does.
//
// Shell-1 classes: when shell 1 joins no sublattice to itself at a non-zero offset, a fewest-
// colour colouring of the sublattices by shell-1 bonds at ANY offset gives classes whose sites never
// bond through shell 1, in every octant at once.  The groups are then numbered class by class
// (each class coloured by the octant rule on its own), so a class is a run of consecutive
// groups; this is kept only when it needs no more groups than the plain octant colouring.
// class_of_group[g] is group g's shell-1 class, or empty when there are no such classes.
namespace {
int greedy_groups(int n, const std::vector<std::vector<char>>& conflict, const std::vector<int>& order,
                  std::vector<int>* colour, int first) {
    int top = first;
    for (int s : order) {
        int g = first;
        for (;; ++g) {
            bool ok = true;
            for (int t = 0; t < n; ++t)
                if ((*colour)[t] == g && conflict[s][t]) { ok = false; break; }
            if (ok) break;
        }
        (*colour)[s] = g;
        top = std::max(top, g + 1);
    }
    return top;
}

// colour the n nodes with k colours by backtracking (a bounded search; false when it finds
// none within the bound)
bool colour_k(int n, const std::vector<std::vector<char>>& conflict, int k, std::vector<int>* colour) {
    colour->assign(n, -1);
    long budget = 1L << 20;
    std::vector<int> next(n, 0);
    int i = 0;
    while (i >= 0 && i < n) {
        if (--budget < 0) return false;
        int c = next[i];
        for (; c < k; ++c) {
            bool ok = true;
            for (int t = 0; t < i; ++t)
                if ((*colour)[t] == c && conflict[i][t]) { ok = false; break; }
            if (ok) break;
        }
        if (c < k) {
            (*colour)[i] = c;
            next[i] = c + 1;
            ++i;
            if (i < n) next[i] = 0;
        } else {
            (*colour)[i] = -1;
            --i;
        }
    }
    return i == n;
}
}  // namespace

bool octant_groups(const Lattice& L, std::vector<int>* group, int* ngroups, std::vector<int>* class_of_group) {
    if ((L.nx & 1) || (L.ny & 1) || (L.nz & 1) || L.nsub > kMaxSub || L.nsub < 1) return false;
    const int n = L.nsub;
    std::vector<std::vector<char>> conflict(n, std::vector<char>(n, 0));
    for (int sh = 0; sh < 2; ++sh)
        for (int s = 0; s < n; ++s)
            for (const NbrSlot& q : L.shell[sh][s]) {
                if ((q.dx & 1) || (q.dy & 1) || (q.dz & 1)) continue;   // different octant
                if (q.sub == s) {
                    if (q.dx || q.dy || q.dz) return false;
                    continue;
                }
                conflict[s][q.sub] = conflict[q.sub][s] = 1;
            }
    std::vector<int> all(n);
    for (int s = 0; s < n; ++s) all[s] = s;
    group->assign(n, -1);
    const int ng = greedy_groups(n, conflict, all, group, 0);
    *ngroups = ng;
    if (class_of_group) class_of_group->clear();
    bool merge = class_of_group != nullptr;
    std::vector<std::vector<char>> bond1(n, std::vector<char>(n, 0));
    for (int s = 0; s < n && merge; ++s)
        for (const NbrSlot& q : L.shell[0][s]) {
            if (q.sub == s) {
                if (q.dx || q.dy || q.dz) { merge = false; break; }
                continue;
            }
            bond1[s][q.sub] = bond1[q.sub][s] = 1;
        }
    if (!merge) return true;
    std::vector<int> cls(n, -1), fewer;
    int nc = greedy_groups(n, bond1, all, &cls, 0);
    for (int k = 1; k < nc; ++k)   // fewer classes than the greedy colouring, where there are
        if (colour_k(n, bond1, k, &fewer)) { cls = fewer; nc = k; break; }
    std::vector<int> g2(n, -1), of;
    int next = 0;
    for (int k = 0; k < nc; ++k) {
        std::vector<int> members;
        for (int s = 0; s < n; ++s)
            if (cls[s] == k) members.push_back(s);
        const int top = greedy_groups(n, conflict, members, &g2, next);
        for (int g = next; g < top; ++g) of.push_back(k);
        next = top;
    }
    if (next > ng) return true;   // the plain octant colouring has fewer groups
    *group = g2;
    *ngroups = next;
    *class_of_group = of;
    return true;
}

// Colour classes of the octant blocks (cell octant o, sublattice s) of an octant-layout
// crystal: block (o, s) reaches block (o', t) through a bond of the active shells from s to t
// at cell offset d when o' = (o + d) & 1 per axis (every extent is even), and two blocks so
// joined get different classes; a bond of a site to itself does not count.  DSatur (Brelaz,
// CACM 22(4), 1979): the next block coloured is the uncoloured one with the most distinct
// colours among its neighbours, ties broken by degree and then by the lower index, and it
// takes the lowest colour free there.  out[k] = the blocks of class k as o * nsub + s,
// ascending; false when a block reaches itself (the octant colouring does not apply).
bool octant_block_classes(const Lattice& L, bool shell2, std::vector<std::vector<int>>* out) {
    const int ns = L.nsub, n = 8 * ns;
    std::vector<std::vector<char>> adj(n, std::vector<char>(n, 0));
    for (int o = 0; o < 8; ++o) {
        const int ox = (o >> 2) & 1, oy = (o >> 1) & 1, oz = o & 1;
        for (int sh = 0; sh < (shell2 ? 2 : 1); ++sh)
            for (int s = 0; s < ns; ++s)
                for (const NbrSlot& q : L.shell[sh][s]) {
                    if (q.sub == s && !q.dx && !q.dy && !q.dz) continue;   // the site itself
                    const int o2 = (((ox + q.dx) & 1) << 2) | (((oy + q.dy) & 1) << 1) | ((oz + q.dz) & 1);
                    const int u = o * ns + s, v = o2 * ns + q.sub;
                    if (u == v) return false;
                    adj[u][v] = adj[v][u] = 1;
                }
    }
    std::vector<int> deg(n, 0), col(n, -1);
    for (int u = 0; u < n; ++u)
        for (int v = 0; v < n; ++v) deg[u] += adj[u][v];
    int ncol = 0;
    for (int step = 0; step < n; ++step) {
        int best = -1, bsat = -1;
        for (int v = 0; v < n; ++v) {
            if (col[v] >= 0) continue;
            std::vector<char> seen(ncol + 1, 0);
            int sat = 0;
            for (int w = 0; w < n; ++w)
                if (adj[v][w] && col[w] >= 0 && !seen[col[w]]) { seen[col[w]] = 1; ++sat; }
            if (sat > bsat || (sat == bsat && deg[v] > deg[best])) { best = v; bsat = sat; }
        }
        std::vector<char> used(ncol + 1, 0);
        for (int w = 0; w < n; ++w)
            if (adj[best][w] && col[w] >= 0) used[col[w]] = 1;
        int c = 0;
        while (used[c]) ++c;
        col[best] = c;
        ncol = std::max(ncol, c + 1);
    }
    out->assign(ncol, {});
    for (int v = 0; v < n; ++v) (*out)[col[v]].push_back(v);
    return true;
}

bool is_checkerboard_sc(const Lattice& L) {
    if (L.nsub != 1) return false;
    if ((L.nx & 1) || (L.ny & 1) || (L.nz & 1)) return false;
    const auto& s = L.shell[0][0];
    if (s.size() != 6) return false;
    int seen = 0;
    for (const auto& q : s) {
        int k = -1;
        if (q.dx == 1 && q.dy == 0 && q.dz == 0) k = 0;
        else if (q.dx == -1 && q.dy == 0 && q.dz == 0) k = 1;
        else if (q.dx == 0 && q.dy == 1 && q.dz == 0) k = 2;
        else if (q.dx == 0 && q.dy == -1 && q.dz == 0) k = 3;
        else if (q.dx == 0 && q.dy == 0 && q.dz == 1) k = 4;
        else if (q.dx == 0 && q.dy == 0 && q.dz == -1) k = 5;
        if (k < 0 || (seen >> k) & 1) return false;
        seen |= 1 << k;
    }
    return seen == 63;
}

}  // namespace isg
