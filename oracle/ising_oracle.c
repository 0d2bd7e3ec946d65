/*
 * ising_oracle.c -- CPU FP64 restatement of the reference path (TEST INFRASTRUCTURE).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline/reference arm load
 * this library; the CUDA product never calls it.  Parity is UNPINNED by the reference
 * (no golden vectors exist upstream and the Fortran cannot be built here); see the
 * header for what pins it instead.
 *
 * Reference files restated (paths within SamuelJosephs/ISING):
 *   src/constants.f90:9-16, src/rand.f90:11-95, src/algo.f90:99-182,353-420,
 *   src/chainMesh.f90:85-241,280-405,495-703,729-911,931-1031,
 *   src/energyMin.f90:49-68,86-229,234-374,499-528,
 *   src/reciprocalSpaceProcesses.f90:284-364,438-500, src/PT.f90:199-272,
 *   src/PT-Utils.f90:33-66, src/LLG.f90:28-73, src/StereographicProjection.f90:58-117.
 */
#include "ising_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ======================= constants ======================= */
/* src/constants.f90:9,11,14,16: default-real literals -> float rounding */
double ora_const_kb(void) { return (double)8.6173303e-5f; }
double ora_const_pi_f(void) { return (double)3.14159265358979323846f; }
double ora_const_g(void) { return 2.0; }
double ora_const_mu_b(void) { return 1.0; }
#define PI_F ((double)3.14159265358979323846f)
#define PI_D 3.14159265358979323846

/* Fortran NINT: round half away from zero */
static long f_nint(double x) { return (long)(x >= 0.0 ? floor(x + 0.5) : -floor(-x + 0.5)); }
/* Fortran MODULO (result has the sign of the divisor) */
static long f_modulo(long a, long p) { long r = a % p; return (r != 0 && ((r < 0) != (p < 0))) ? r + p : r; }

/* ======================= reference RNG ======================= */
/* makeRandom (src/rand.f90:11-18) */
ora_random ora_make_random(int32_t seed)
{
    ora_random o;
    o.seed = seed;
    o.ix = (int32_t)(777755555u ^ (uint32_t)seed);
    o.iy = (int32_t)((888889999u ^ (uint32_t)seed) | 1u);
    return o;
}

/* algor_uniform_random (src/rand.f90:19-95): Marsaglia xorshift (13,-17,5) with logical
 * shifts (ishft), Park-Miller with Schrage's factorisation, combined and masked to (0,1]. */
double ora_uniform(ora_random* r)
{
    uint32_t ix = (uint32_t)r->ix;
    ix ^= ix << 13;
    ix ^= ix >> 17;
    ix ^= ix << 5;
    int32_t iy = r->iy;
    int32_t iy_tmp = iy / 127773;
    iy = 16807 * (iy - iy_tmp * 127773) - iy_tmp * 2836;
    if (iy < 0) iy += 2147483647;
    int32_t comb = (int32_t)((2147483647u & (ix ^ (uint32_t)iy)) | 1u);
    r->ix = (int32_t)ix;
    r->iy = iy;
    return (1.0 / 2147483647.0) * (double)comb;
}

void ora_uniform_stream(int32_t seed, int n, double* out)
{
    ora_random r = ora_make_random(seed);
    for (int i = 0; i < n; ++i) out[i] = ora_uniform(&r);
}

/* ======================= Philox4x32 ======================= */
/* Counter-based generator of Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
 * as 1, 2, 3" (SC'11): per round (hi,lo) of two 32x32 products, S-box mixing and a Weyl key
 * schedule.  Multipliers and Weyl increments are the published ones. */
void ora_philox4x32(const uint32_t ctr[4], const uint32_t key[2], int rounds, uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int i = 0; i < rounds; ++i) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

double ora_u01(uint32_t x) { return (double)(2u * (x >> 9) + 1u) * (1.0 / 16777216.0); }

/* Counter layout shared with the CUDA product:
 *   ctr = (site, sweep, replica, ensemble<<8 | tag), key = (seed lo, seed hi).
 *   tag 0: sweep trial, 1: initial spins, 2: replica exchange. */
static void philox_draw(uint64_t seed, uint32_t site, uint32_t sweep, uint32_t replica,
                        uint32_t ensemble, uint32_t tag, int rounds, double u[4])
{
    uint32_t ctr[4] = {site, sweep, replica, (ensemble << 8) | (tag & 0xffu)};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t o[4];
    ora_philox4x32(ctr, key, rounds, o);
    for (int i = 0; i < 4; ++i) u[i] = ora_u01(o[i]);
}

/* ======================= mergesort (src/algo.f90:99-182, 353-420) ======================= */
/* Bottom-up pairwise merge; merge_dp takes A(1) only when A(1) < B(1), so on ties the
 * right run's element comes first.  Restated so neighbour order matches the reference. */
static void ref_mergesort(double* a, int* comp, int n)
{
    if (n <= 1) return;
    int* lo = malloc(sizeof(int) * n);
    int* hi = malloc(sizeof(int) * n);
    double* sa = malloc(sizeof(double) * n);
    int* sc = malloc(sizeof(int) * n);
    int nb = n;
    for (int i = 0; i < n; ++i) { lo[i] = i; hi[i] = i; }
    while (nb > 1) {
        int cnt = 0;
        int pairs = nb / 2;
        for (int i = 0; i < pairs; ++i) {
            int a0 = lo[2 * i], a1 = hi[2 * i], b0 = lo[2 * i + 1], b1 = hi[2 * i + 1];
            int ia = a0, ib = b0, k = 0;
            while (ia <= a1 && ib <= b1) {
                if (a[ia] < a[ib]) { sa[k] = a[ia]; sc[k] = comp[ia]; ++ia; }
                else { sa[k] = a[ib]; sc[k] = comp[ib]; ++ib; }
                ++k;
            }
            while (ia <= a1) { sa[k] = a[ia]; sc[k] = comp[ia]; ++ia; ++k; }
            while (ib <= b1) { sa[k] = a[ib]; sc[k] = comp[ib]; ++ib; ++k; }
            memcpy(a + a0, sa, sizeof(double) * k);
            memcpy(comp + a0, sc, sizeof(int) * k);
            lo[cnt] = a0; hi[cnt] = b1; ++cnt;
        }
        if (nb % 2) { lo[cnt] = lo[nb - 1]; hi[cnt] = hi[nb - 1]; ++cnt; }
        nb = cnt;
    }
    free(lo); free(hi); free(sa); free(sc);
}

/* ======================= lattice ======================= */
struct ora_mesh {
    int nx, ny, nz, nsub, nshells;
    long ncells, natoms;
    double a, b, c;
    double av[3], bv[3], cv[3], ar[3], br[3], cr[3];
    float *x, *y, *z;            /* Atom_t%x,y,z are real(4) (src/atom.f90:5) */
    int* first_atom;             /* ChainMeshCell_t%firstAtomInMeshCell */
    int* next_atom;              /* Atom_t%nextAtom */
    int* sh_off;                 /* (natoms*nshells + 1) offsets into sh_idx */
    int* sh_idx;
    int* nl_off;                 /* legacy NeighborList CSR */
    int* nl_idx;
    int* deriv;                  /* [atom][d][side] */
    double* spins;               /* atomSpins(numAtoms,3), column-major */
};

long ora_mesh_natoms(const ora_mesh* m) { return m->natoms; }
double* ora_mesh_spins(ora_mesh* m) { return m->spins; }
int ora_mesh_first_atom(const ora_mesh* m, long cell) { return m->first_atom[cell]; }

void ora_mesh_vectors(const ora_mesh* m, double out[18])
{
    memcpy(out, m->av, 24); memcpy(out + 3, m->bv, 24); memcpy(out + 6, m->cv, 24);
    memcpy(out + 9, m->ar, 24); memcpy(out + 12, m->br, 24); memcpy(out + 15, m->cr, 24);
}

void ora_mesh_positions(const ora_mesh* m, float* xyz)
{
    for (long i = 0; i < m->natoms; ++i) {
        xyz[3 * i] = m->x[i]; xyz[3 * i + 1] = m->y[i]; xyz[3 * i + 2] = m->z[i];
    }
}

static void cross3(const double a[3], const double b[3], double o[3])
{
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}
static double dot3(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* coordinatesFromIndex (src/chainMesh.f90:687-703), 0-based */
static void cell_coords(const ora_mesh* m, long cell, int* i, int* j, int* k)
{
    long bc = (long)m->ny * m->nz;
    *i = (int)(cell / bc);
    long rem = cell % bc;
    *j = (int)(rem / m->nz);
    *k = (int)(rem % m->nz);
}
/* IndexFromCoordinatesInteger (src/chainMesh.f90:673-685), 0-based */
static long cell_index(const ora_mesh* m, int i, int j, int k)
{
    return ((long)i * m->ny + j) * m->nz + k;
}

/* min-image Bravais coefficients of r_j - r_i (distance_points_vec_bravais, :244-276) */
static void min_image_coeff(const ora_mesh* m, long i, long j, double co[3])
{
    double dx = (double)m->x[j] - (double)m->x[i];
    double dy = (double)m->y[j] - (double)m->y[i];
    double dz = (double)m->z[j] - (double)m->z[i];
    double ac = dx * m->ar[0] + dy * m->ar[1] + dz * m->ar[2];
    double bc = dx * m->br[0] + dy * m->br[1] + dz * m->br[2];
    double cc = dx * m->cr[0] + dy * m->cr[1] + dz * m->cr[2];
    double wx = (double)m->nx, wy = (double)m->ny, wz = (double)m->nz;
    co[0] = ac - wx * (double)f_nint(ac / wx);
    co[1] = bc - wy * (double)f_nint(bc / wy);
    co[2] = cc - wz * (double)f_nint(cc / wz);
}

/* distance_points_vec (:206-241) */
void ora_mesh_min_image(const ora_mesh* m, long i, long j, double out[3])
{
    double co[3];
    min_image_coeff(m, i, j, co);
    for (int d = 0; d < 3; ++d) out[d] = co[0] * m->av[d] + co[1] * m->bv[d] + co[2] * m->cv[d];
}

/* distance (:133-169): the coordinate differences are taken between real(4) fields
 * (single-precision subtraction, :151-153) and the result is real(4). */
static float atom_distance(const ora_mesh* m, long i, long j)
{
    double dx = (double)(m->x[j] - m->x[i]);
    double dy = (double)(m->y[j] - m->y[i]);
    double dz = (double)(m->z[j] - m->z[i]);
    double ac = dx * m->ar[0] + dy * m->ar[1] + dz * m->ar[2];
    double bc = dx * m->br[0] + dy * m->br[1] + dz * m->br[2];
    double cc = dx * m->cr[0] + dy * m->cr[1] + dz * m->cr[2];
    ac = ac - (double)m->nx * (double)f_nint(ac / (double)m->nx);
    bc = bc - (double)m->ny * (double)f_nint(bc / (double)m->ny);
    cc = cc - (double)m->nz * (double)f_nint(cc / (double)m->nz);
    double r[3];
    for (int d = 0; d < 3; ++d) r[d] = ac * m->av[d] + bc * m->bv[d] + cc * m->cv[d];
    return (float)sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
}

/* getNeighboringCells (:85-131): 27 cells, wrap at -1 and N only */
static void neighboring_cells(const ora_mesh* m, long cell, long out[27])
{
    int ic, jc, kc, n = 0;
    cell_coords(m, cell, &ic, &jc, &kc);
    for (int i = ic - 1; i <= ic + 1; ++i)
        for (int j = jc - 1; j <= jc + 1; ++j)
            for (int k = kc - 1; k <= kc + 1; ++k) {
                int it = i, jt = j, kt = k;
                if (it == m->nx) it = 0; else if (it == -1) it = m->nx - 1;
                if (jt == m->ny) jt = 0; else if (jt == -1) jt = m->ny - 1;
                if (kt == m->nz) kt = 0; else if (kt == -1) kt = m->nz - 1;
                out[n++] = cell_index(m, it, jt, kt);
            }
}

/* assignNearestNeighbors / AssignAtomNearestNeighbhors (:280-405): legacy NeighborList */
static void assign_nearest_neighbors(ora_mesh* m)
{
    int cap = 27 * m->nsub + 1;
    int* cnt = calloc((size_t)m->natoms, sizeof(int));
    int** lists = calloc((size_t)m->natoms, sizeof(int*));
    /* atoms are independent: the reference serialises this loop with !$omp critical */
#pragma omp parallel
    {
    int* tmp = malloc(sizeof(int) * cap);
    long nbc[27];
#pragma omp for schedule(static)
    for (long idex = 0; idex < m->ncells; ++idex) {
        neighboring_cells(m, idex, nbc);
        for (int at = m->first_atom[idex]; at != -1; at = m->next_atom[at]) {
            float nnd = 3.4028235e38f; /* HUGE(0.0) */
            for (int c = 0; c < 27; ++c)
                for (int t = m->first_atom[nbc[c]]; t != -1; t = m->next_atom[t]) {
                    if (t == at) continue;
                    float d = atom_distance(m, at, t);
                    if (d < nnd) nnd = d;
                }
            int n = 0;
            for (int c = 0; c < 27; ++c)
                for (int t = m->first_atom[nbc[c]]; t != -1; t = m->next_atom[t]) {
                    if (t == at) continue;
                    int dup = 0;
                    for (int q = 0; q < n; ++q) if (tmp[q] == t) { dup = 1; break; }
                    if (dup) continue;
                    float d = atom_distance(m, at, t);
                    if (fabs((double)(d - nnd)) < m->a / 100.0) tmp[n++] = t;
                }
            lists[at] = malloc(sizeof(int) * (n > 0 ? n : 1));
            memcpy(lists[at], tmp, sizeof(int) * n);
            cnt[at] = n;
        }
    }
    free(tmp);
    }
    m->nl_off = malloc(sizeof(int) * (m->natoms + 1));
    m->nl_off[0] = 0;
    for (long i = 0; i < m->natoms; ++i) m->nl_off[i + 1] = m->nl_off[i] + cnt[i];
    m->nl_idx = malloc(sizeof(int) * (m->nl_off[m->natoms] + 1));
    for (long i = 0; i < m->natoms; ++i) {
        memcpy(m->nl_idx + m->nl_off[i], lists[i], sizeof(int) * cnt[i]);
        free(lists[i]);
    }
    free(lists); free(cnt);
}

/* NNearestCells (:593-635) and initAtomShells (:495-591) */
static void init_atom_shells(ora_mesh* m, int N, double thr)
{
    int ncell_list = (2 * N + 1) * (2 * N + 1) * (2 * N + 1);
    int cap = ncell_list * m->nsub;
    /* per (atom, shell) counts then lists; store as growable per-atom buffers */
    int* sizes = calloc((size_t)m->natoms * N, sizeof(int));
    int** lists = calloc((size_t)m->natoms, sizeof(int*));
#pragma omp parallel
    {
    double* dist = malloc(sizeof(double) * cap);
    int* idx = malloc(sizeof(int) * cap);
    long* clist = malloc(sizeof(long) * ncell_list);
    int* shell_of = malloc(sizeof(int) * cap);
#pragma omp for schedule(static)
    for (long cell = 0; cell < m->ncells; ++cell) {
        int ac, bc, cc, n = 0;
        cell_coords(m, cell, &ac, &bc, &cc);
        for (int i = -N; i <= N; ++i)
            for (int j = -N; j <= N; ++j)
                for (int k = -N; k <= N; ++k)
                    clist[n++] = cell_index(m, (int)f_modulo(ac + i, m->nx),
                                            (int)f_modulo(bc + j, m->ny),
                                            (int)f_modulo(cc + k, m->nz));
        for (int at = m->first_atom[cell]; at != -1; at = m->next_atom[at]) {
            int nd = 0;
            for (int q = 0; q < cap; ++q) { dist[q] = 1.7976931348623157e308; idx[q] = -1; }
            for (int q = 0; q < ncell_list; ++q)
                for (int t = m->first_atom[clist[q]]; t != -1; t = m->next_atom[t]) {
                    if (t == at) continue;
                    dist[nd] = (double)atom_distance(m, at, t);
                    idx[nd] = t;
                    ++nd;
                }
            ref_mergesort(dist, idx, cap);
            int shell = 0, total = 0;
            shell_of[total++] = 0;
            for (int q = 1; q < cap; ++q) {
                if (idx[q] < 0) break; /* padding (HUGE) entries: lattice too small */
                if (fabs(dist[q] - dist[q - 1]) > thr) ++shell;
                if (shell >= N) break;
                shell_of[total++] = shell;
            }
            lists[at] = malloc(sizeof(int) * (total + 1));
            /* group by shell preserving order */
            int w = 0;
            for (int s = 0; s < N; ++s)
                for (int q = 0; q < total; ++q)
                    if (shell_of[q] == s) { lists[at][w++] = idx[q]; ++sizes[(long)at * N + s]; }
        }
    }
    free(dist); free(idx); free(clist); free(shell_of);
    }
    m->sh_off = malloc(sizeof(int) * ((size_t)m->natoms * N + 1));
    m->sh_off[0] = 0;
    for (long q = 0; q < m->natoms * N; ++q) m->sh_off[q + 1] = m->sh_off[q] + sizes[q];
    m->sh_idx = malloc(sizeof(int) * (m->sh_off[m->natoms * N] + 1));
    for (long at = 0; at < m->natoms; ++at) {
        int tot = m->sh_off[(at + 1) * N] - m->sh_off[at * N];
        memcpy(m->sh_idx + m->sh_off[at * N], lists[at], sizeof(int) * tot);
        free(lists[at]);
    }
    free(lists); free(sizes);
}

/* DerivativeList / computeAdjacentAtoms (:931-1031).  Returns 0 on success, -1 if an atom
 * has no neighbour on one side ("Unable to locate atoms", :1028). */
static int derivative_list(ora_mesh* m)
{
    m->deriv = malloc(sizeof(int) * m->natoms * 6);
    long nbc[27];
    for (int d = 0; d < 3; ++d)
        for (long cell = 0; cell < m->ncells; ++cell) {
            neighboring_cells(m, cell, nbc);
            for (int at = m->first_atom[cell]; at != -1; at = m->next_atom[at]) {
                int imin = -1, imax = -1;
                double cmin = 1.7976931348623157e308, cmax = 1.7976931348623157e308;
                for (int c = 0; c < 27; ++c) {
                    if (nbc[c] == cell) continue;
                    for (int t = m->first_atom[nbc[c]]; t != -1; t = m->next_atom[t]) {
                        if (t == at) continue;
                        double co[3];
                        min_image_coeff(m, at, t, co);
                        int cand = 1;
                        for (int j = 0; j < 3; ++j) {
                            if (j == d) continue;
                            if (fabs(co[j]) > 0.0001) { cand = 0; break; }
                        }
                        if (!cand) continue;
                        if (co[d] < 0.0 && fabs(co[d]) <= cmin) { cmin = fabs(co[d]); imin = t; }
                        if (co[d] > 0.0 && fabs(co[d]) <= cmax) { cmax = fabs(co[d]); imax = t; }
                    }
                }
                if (imin == -1 || imax == -1) return -1;
                m->deriv[(long)at * 6 + d * 2 + 0] = imin;
                m->deriv[(long)at * 6 + d * 2 + 1] = imax;
            }
        }
    return 0;
}

int ora_mesh_deriv(const ora_mesh* m, long atom, int d, int side) { return m->deriv[atom * 6 + d * 2 + side]; }

int ora_mesh_shell_size(const ora_mesh* m, long atom, int shell)
{
    long q = atom * m->nshells + shell;
    return m->sh_off[q + 1] - m->sh_off[q];
}
int ora_mesh_shell_list(const ora_mesh* m, long atom, int shell, int* out)
{
    long q = atom * m->nshells + shell;
    int n = m->sh_off[q + 1] - m->sh_off[q];
    memcpy(out, m->sh_idx + m->sh_off[q], sizeof(int) * n);
    return n;
}
int ora_mesh_nl_size(const ora_mesh* m, long atom) { return m->nl_off[atom + 1] - m->nl_off[atom]; }
int ora_mesh_nl_list(const ora_mesh* m, long atom, int* out)
{
    int n = m->nl_off[atom + 1] - m->nl_off[atom];
    memcpy(out, m->nl_idx + m->nl_off[atom], sizeof(int) * n);
    return n;
}

/* makeChainMesh (:729-911) without the FFT plans (demag is out of scope) */
ora_mesh* ora_mesh_create(const float* frac, int nsub, int nx, int ny, int nz,
                          double a, double b, double c, double ab_deg, double bc_deg,
                          double ca_deg, double shell_tol, int n_shells)
{
    if (nsub < 1 || nx < 1 || ny < 1 || nz < 1) return NULL;
    ora_mesh* m = calloc(1, sizeof(ora_mesh));
    double thr = shell_tol > 0.0 ? shell_tol : 0.1 * a;   /* :783,785 */
    int N = n_shells > 0 ? n_shells : 2;                    /* :784,786 */
    m->nx = nx; m->ny = ny; m->nz = nz; m->nsub = nsub; m->nshells = N;
    m->a = a; m->b = b; m->c = c;
    double ab = ab_deg * (PI_F / 180.0), bc = bc_deg * (PI_F / 180.0), ca = ca_deg * (PI_F / 180.0);
    m->av[0] = a; m->av[1] = 0.0; m->av[2] = 0.0;                       /* :798 */
    m->bv[0] = b * cos(ab); m->bv[1] = b * sin(ab); m->bv[2] = 0.0;     /* :799 */
    double cx = c * cos(ca);                                            /* :800 */
    double cy = (c * b * cos(bc) - cx * m->bv[0]);                      /* :801 (no /b_y) */
    double cz = sqrt(c * c - cx * cx - cy * cy);                        /* :802 */
    m->cv[0] = cx; m->cv[1] = cy; m->cv[2] = cz;
    for (int d = 0; d < 3; ++d) {                                       /* :813-815 */
        if (!(fabs(m->av[d]) > 1e-5)) m->av[d] = 0.0;
        if (!(fabs(m->bv[d]) > 1e-5)) m->bv[d] = 0.0;
        if (!(fabs(m->cv[d]) > 1e-5)) m->cv[d] = 0.0;
    }
    double t[3];                                                        /* :823-825 */
    cross3(m->bv, m->cv, t); { double s = dot3(m->av, t); for (int d = 0; d < 3; ++d) m->ar[d] = t[d] / s; }
    cross3(m->cv, m->av, t); { double s = dot3(m->bv, t); for (int d = 0; d < 3; ++d) m->br[d] = t[d] / s; }
    cross3(m->av, m->bv, t); { double s = dot3(m->cv, t); for (int d = 0; d < 3; ++d) m->cr[d] = t[d] / s; }

    m->ncells = (long)nx * ny * nz;
    m->natoms = m->ncells * nsub;
    m->x = malloc(sizeof(float) * m->natoms);
    m->y = malloc(sizeof(float) * m->natoms);
    m->z = malloc(sizeof(float) * m->natoms);
    m->first_atom = malloc(sizeof(int) * m->ncells);
    m->next_atom = malloc(sizeof(int) * m->natoms);
    for (long j = 0; j < m->ncells; ++j) {                              /* :853-882 */
        m->first_atom[j] = -1;
        int ic, jc, kc;
        cell_coords(m, j, &ic, &jc, &kc);
        double tv[3];
        for (int d = 0; d < 3; ++d)
            tv[d] = m->av[d] * (double)ic + m->bv[d] * (double)jc + m->cv[d] * (double)kc;
        for (int i = 0; i < nsub; ++i) {
            double fx = (double)frac[3 * i], fy = (double)frac[3 * i + 1], fz = (double)frac[3 * i + 2];
            double pos[3];
            for (int d = 0; d < 3; ++d) pos[d] = fx * m->av[d] + fy * m->bv[d] + fz * m->cv[d];
            long at = j * nsub + i;
            m->x[at] = (float)(pos[0] + tv[0]);
            m->y[at] = (float)(pos[1] + tv[1]);
            m->z[at] = (float)(pos[2] + tv[2]);
            m->next_atom[at] = m->first_atom[j];                        /* addAtomToChainCell :663-671 */
            m->first_atom[j] = (int)at;
        }
    }
    assign_nearest_neighbors(m);                                        /* :884 */
    m->spins = calloc((size_t)m->natoms * 3, sizeof(double));           /* :889 (uninitialised there) */
    if (derivative_list(m) != 0) { ora_mesh_destroy(m); return NULL; }   /* :891 */
    init_atom_shells(m, N, thr);                                        /* :892 */
    return m;
}

void ora_mesh_destroy(ora_mesh* m)
{
    if (!m) return;
    free(m->x); free(m->y); free(m->z); free(m->first_atom); free(m->next_atom);
    free(m->sh_off); free(m->sh_idx); free(m->nl_off); free(m->nl_idx); free(m->deriv);
    free(m->spins); free(m);
}

/* ======================= energies ======================= */
static void get_spin(const ora_mesh* m, long i, double s[3])
{
    s[0] = m->spins[i]; s[1] = m->spins[m->natoms + i]; s[2] = m->spins[2 * m->natoms + i];
}

/* D vector for the bond i->j as the local routine builds it (energyMin.f90:114,135-138):
 * r = -(r_j - r_i)_min / |.|, D = Dz * axis x r (interfacial) or Dz * r (bulk). */
static void bond_dmi(const ora_mesh* m, long i, long j, double Dz, const double axis[3],
                     int bulk, double D[3])
{
    double r[3];
    ora_mesh_min_image(m, i, j, r);
    double n = sqrt(dot3(r, r));
    for (int d = 0; d < 3; ++d) r[d] = -r[d] / n;
    if (bulk) { for (int d = 0; d < 3; ++d) D[d] = Dz * r[d]; }
    else {
        double tv[3] = {Dz * axis[0], Dz * axis[1], Dz * axis[2]};
        cross3(tv, r, D);
    }
}

static double aniso(const ora_params* p, const double s[3])
{
    if (p->K == 0.0) return 0.0;
    double d = dot3(s, p->K_axis);
    return -p->K * d * d;
}

/* calculateHeisenbergEnergy (energyMin.f90:86-171), demag disabled (:163-167 skipped). */
void ora_local_energy(const ora_mesh* m, long at, const ora_params* p,
                      const double sp[3], double* old_e, double* new_e)
{
    double S[3], Sj[3], D[3], cr[3];
    get_spin(m, at, S);
    double cn = sqrt(dot3(m->cv, m->cv));
    double axis[3] = {m->cv[0] / cn, m->cv[1] / cn, m->cv[2] / cn};   /* Dz*(c_vec/|c_vec|), :114 */
    double oe = 0.0, ne = 0.0;
    int n1 = ora_mesh_shell_size(m, at, 0);
    const int* l1 = m->sh_idx + m->sh_off[at * m->nshells];
    for (int q = 0; q < n1; ++q) {                                   /* :122-142 */
        long j = l1[q];
        get_spin(m, j, Sj);
        bond_dmi(m, at, j, p->Dz, axis, p->dmi_bulk, D);
        cross3(S, Sj, cr);
        oe = oe + (p->J * dot3(S, Sj) + dot3(D, cr));
        cross3(sp, Sj, cr);
        ne = ne + (p->J * dot3(sp, Sj) + dot3(D, cr));
    }
    if (m->nshells > 1) {                                            /* :145-157 */
        int n2 = ora_mesh_shell_size(m, at, 1);
        const int* l2 = m->sh_idx + m->sh_off[at * m->nshells + 1];
        for (int q = 0; q < n2; ++q) {
            get_spin(m, l2[q], Sj);
            oe = oe + p->J_prime * dot3(S, Sj);
            ne = ne + p->J_prime * dot3(sp, Sj);
        }
    }
    oe = oe - p->B * S[2];                                           /* :161-162 */
    ne = ne - p->B * sp[2];
    oe += aniso(p, S);
    ne += aniso(p, sp);
    *old_e = oe; *new_e = ne;
}

/* TotalHeisenbergEnergy (:499-528) + helper (:174-229): legacy NeighborList, D axis z,
 * 0.5 per bond, -g mu_B B S_z, no J'. */
double ora_total_energy(const ora_mesh* m, const ora_params* p, double zeeman_gmu)
{
    const double zaxis[3] = {0.0, 0.0, 1.0};
    double tot = 0.0;
    for (long at = 0; at < m->natoms; ++at) {
        double S[3], Sj[3], D[3], cr[3], e = 0.0;
        get_spin(m, at, S);
        for (int q = m->nl_off[at]; q < m->nl_off[at + 1]; ++q) {
            long j = m->nl_idx[q];
            get_spin(m, j, Sj);
            bond_dmi(m, at, j, p->Dz, zaxis, p->dmi_bulk, D);
            cross3(S, Sj, cr);
            e = e + 0.5 * ((p->J * dot3(S, Sj)) + dot3(D, cr));
        }
        e = e - (zeeman_gmu * p->B * S[2]);
        e += aniso(p, S);
        tot = tot + e;
    }
    return tot;
}

double ora_canonical_energy(const ora_mesh* m, const ora_params* p)
{
    double cn = sqrt(dot3(m->cv, m->cv));
    double axis[3] = {m->cv[0] / cn, m->cv[1] / cn, m->cv[2] / cn};
    double tot = 0.0;
    for (long at = 0; at < m->natoms; ++at) {
        double S[3], Sj[3], D[3], cr[3], e = 0.0;
        get_spin(m, at, S);
        for (int s = 0; s < m->nshells && s < 2; ++s) {
            long q0 = m->sh_off[at * m->nshells + s], q1 = m->sh_off[at * m->nshells + s + 1];
            for (long q = q0; q < q1; ++q) {
                long j = m->sh_idx[q];
                get_spin(m, j, Sj);
                if (s == 0) {
                    bond_dmi(m, at, j, p->Dz, axis, p->dmi_bulk, D);
                    cross3(S, Sj, cr);
                    e += 0.5 * (p->J * dot3(S, Sj) + dot3(D, cr));
                } else {
                    e += 0.5 * p->J_prime * dot3(S, Sj);
                }
            }
        }
        e -= p->B * S[2];
        e += aniso(p, S);
        tot += e;
    }
    return tot;
}

/* ======================= winding number ======================= */
/* arc_winding (rsp:284-318): Berg-Luscher signed area 2*atan2(Im, Re) of
 * (1 + s1.s2 + s2.s3 + s3.s1 + i s1.(s2 x s3)) / sqrt(2(1+s1.s2)(1+s2.s3)(1+s3.s1)). */
double ora_arc_winding(const double s1[3], const double s2[3], const double s3[3])
{
    double c23[3];
    cross3(s2, s3, c23);
    double re = 1.0 + dot3(s1, s2) + dot3(s2, s3) + dot3(s3, s1);
    double im = dot3(s1, c23);
    double nrm = sqrt(2.0 * (1.0 + dot3(s1, s2)) * (1.0 + dot3(s2, s3)) * (1.0 + dot3(s3, s1)));
    re = re / nrm;
    im = im / nrm;
    return 2.0 * atan2(im, re);
}

static void unit_spin(const ora_mesh* m, long i, double s[3])
{
    get_spin(m, i, s);
    double n = sqrt(dot3(s, s));
    s[0] /= n; s[1] /= n; s[2] /= n;
}

static double plaquette(const ora_mesh* m, int i, int j, int zc)
{
    long cell = cell_index(m, i, j, zc);
    long a1 = m->first_atom[cell];
    long a2 = m->deriv[a1 * 6 + 0 * 2 + 1];
    long a4 = m->deriv[a2 * 6 + 1 * 2 + 1];
    long a3 = m->deriv[a1 * 6 + 1 * 2 + 1];
    double s1[3], s2[3], s3[3], s4[3];
    unit_spin(m, a1, s1); unit_spin(m, a2, s2); unit_spin(m, a3, s3); unit_spin(m, a4, s4);
    return ora_arc_winding(s1, s2, s4) + ora_arc_winding(s1, s4, s3);
}

/* calculate_winding_number2 (rsp:320-364) */
double ora_winding_number(const ora_mesh* m, int z1)
{
    if (z1 < 1 || z1 > m->nz) return NAN;
    double w = 0.0;
    for (int i = 0; i < m->nx; ++i)
        for (int j = 0; j < m->ny; ++j) w = w + plaquette(m, i, j, z1 - 1);
    return w / (4.0 * PI_F);
}

/* calculate_winding_number_density (rsp:438-500) */
void ora_winding_density(const ora_mesh* m, int z1, double* dens)
{
    for (int i = 0; i < m->nx; ++i)
        for (int j = 0; j < m->ny; ++j)
            dens[i + (long)j * m->nx] = plaquette(m, i, j, z1 - 1) / (4.0 * PI_F);
}

/* chainMesh_statistics (PT-Utils.f90:33-66), skyrmion count omitted */
void ora_statistics(const ora_mesh* m, double* wnd_mid, double* wnd_spread, double mag[3])
{
    double mx = -1.7976931348623157e308, mn = 1.7976931348623157e308;
    for (int z = 1; z <= m->nz; ++z) {
        double w = ora_winding_number(m, z);
        if (w > mx) mx = w;
        if (w < mn) mn = w;
        if (z == m->nz / 2) *wnd_mid = w;
    }
    *wnd_spread = fabs(mx - mn);
    double s[3] = {0, 0, 0};
    for (long i = 0; i < m->natoms; ++i) {
        s[0] += m->spins[i]; s[1] += m->spins[m->natoms + i]; s[2] += m->spins[2 * m->natoms + i];
    }
    for (int d = 0; d < 3; ++d) mag[d] = s[d] / (double)m->natoms;
}

/* ======================= skyrmion counting ======================= */
/* Fine-grid arrays are column-major (first index fastest), 1-based in the comments as in the
 * reference.  The summations below are written without fused multiply-adds so that their
 * rounding is defined by the order alone. */
#define IDX2(a, i, j, ld) (a)[((long)(i) - 1) + ((long)(j) - 1) * (long)(ld)]

/* Gaussian_filter_2d (rsp:814-859): 5x5 kernel exp(-(di^2+dj^2)/(2 sigma^2)) normalised by
 * its sum; buffer(i,j) = sum_{l,m=1..5} array(i-l, j-m) G(l,m) with periodic indices
 * (index 0 -> Nx, -k -> Nx-k), l outer and m inner.  The output is shifted by 3 cells
 * against a centred filter, as in the reference.  Requires nx, ny >= 5. */
__attribute__((optimize("fp-contract=off")))
void ora_gaussian_kernel(double sigma, double G[25])
{
    const int k = 2;
    double acc = 0.0;
    for (int i = 1; i <= 2 * k + 1; ++i)
        for (int j = 1; j <= 2 * k + 1; ++j) {
            const int num = (i - k - 1) * (i - k - 1) + (j - k - 1) * (j - k - 1);
            const double g = exp((double)(-num) / (2.0 * (sigma * sigma)));
            G[(i - 1) * 5 + (j - 1)] = g;
            acc = acc + g;
        }
    for (int q = 0; q < 25; ++q) G[q] = G[q] / acc;
}

__attribute__((optimize("fp-contract=off")))
int ora_gaussian_filter_2d(double* a, int nx, int ny, double sigma)
{
    if (nx < 5 || ny < 5) return 1;
    double G[25];
    ora_gaussian_kernel(sigma, G);
    double* buf = (double*)calloc((size_t)nx * ny, sizeof(double));
    if (!buf) return 2;
    for (int i = 1; i <= nx; ++i)
        for (int j = 1; j <= ny; ++j) {
            double acc = 0.0;
            for (int l = 1; l <= 5; ++l)
                for (int m = 1; m <= 5; ++m) {
                    int ii = i - l, jj = j - m;
                    if (ii > nx) ii -= nx;
                    if (ii < 1) ii = nx - abs(ii);
                    if (jj > ny) jj -= ny;
                    if (jj < 1) jj = ny - abs(jj);
                    const double t = IDX2(a, ii, jj, nx) * G[(l - 1) * 5 + (m - 1)];
                    acc = acc + t;
                }
            IDX2(buf, i, j, nx) = acc;
        }
    memcpy(a, buf, sizeof(double) * (size_t)nx * ny);
    free(buf);
    return 0;
}

/* add_neighbors_to_stack (rsp:582-622): the 3x3 neighbourhood of (i,j) wrapped with the
 * COARSE cell counts ncx, ncy (index < 1 -> ncx, index > ncx -> 1); an unvisited, masked,
 * not-yet-stacked, downhill neighbour is pushed.  Returns 1 when the 10000-row stack would
 * overflow ("Stack array capacity exceeded"). */
static int sk_push_neighbours(int i, int j, int ncx, int ncy, int fx, int* stack, int* sp,
                              const unsigned char* visited, const unsigned char* mask,
                              unsigned char* in_stack, const double* d)
{
    const double dij = fabs(IDX2(d, i, j, fx));
    for (int di = -1; di <= 1; ++di)
        for (int dj = -1; dj <= 1; ++dj) {
            int it = i + di, jt = j + dj;
            if (it < 1) it = ncx;
            if (it > ncx) it = 1;
            if (jt < 1) jt = ncy;
            if (jt > ncy) jt = 1;
            if (IDX2(in_stack, it, jt, fx)) continue;
            const int downhill = dij >= fabs(IDX2(d, it, jt, fx)) - 1e-10;
            if (!IDX2(visited, it, jt, fx) && IDX2(mask, it, jt, fx) && downhill) {
                if (*sp + 1 > 10000) return 1;
                stack[2 * (*sp - 1)] = it;
                stack[2 * (*sp - 1) + 1] = jt;
                *sp += 1;
                IDX2(in_stack, it, jt, fx) = 1;
            }
        }
    return 0;
}

/* calculate_skyrmion_number (rsp:627-812) after its interpolation step: dens is the fx x fy
 * fine-grid density (overwritten by its Gaussian-filtered copy), ncx x ncy the coarse cell
 * counts that the reference uses for every periodic wrap.  Status 0, 1 on a q_threshold
 * outside [0,1], 2 on stack overflow, 3 on a fine grid below 5x5, 4 on allocation failure. */
__attribute__((optimize("fp-contract=off")))
int ora_skyrmion_number(double* d, int fx, int fy, int ncx, int ncy, double q_threshold,
                        int particle_number, double sigma, int* out)
{
    const double skThreshold = 0.05;
    if (fabs(q_threshold) > 1.0 || q_threshold < 0.0) return 1;
    if (ora_gaussian_filter_2d(d, fx, fy, sigma)) return 3;
    const long n = (long)fx * fy;
    double mx = 0.0;
    for (long q = 0; q < n; ++q) if (fabs(d[q]) > mx) mx = fabs(d[q]);
    unsigned char* mask = (unsigned char*)malloc(n);
    unsigned char* visited = (unsigned char*)calloc(n, 1);
    unsigned char* in_stack = (unsigned char*)calloc(n, 1);
    int* region = (int*)calloc(n, sizeof(int));
    int* stack = (int*)malloc(sizeof(int) * 2 * 10000);
    long cap = 64, nreg = 0;
    double* accs = (double*)malloc(sizeof(double) * cap);
    unsigned char* merged = (unsigned char*)malloc(cap);
    int status = 0;
    if (!mask || !visited || !in_stack || !region || !stack || !accs || !merged) { status = 4; goto done; }
    for (long q = 0; q < n; ++q) mask[q] = fabs(d[q]) > q_threshold * mx;
    for (int i = 1; i <= fx && !status; ++i)
        for (int j = 1; j <= fy && !status; ++j) {
            int is_max = 1;
            for (int di = -1; di <= 1; ++di)
                for (int dj = -1; dj <= 1; ++dj) {
                    const int x = (int)f_modulo(i + di - 1, ncx) + 1, y = (int)f_modulo(j + dj - 1, ncy) + 1;
                    if (di == 0 && dj == 0) continue;
                    if (fabs(IDX2(d, i, j, fx)) < fabs(IDX2(d, x, y, fx))) is_max = 0;
                }
            if (!(IDX2(mask, i, j, fx) && !IDX2(visited, i, j, fx) && is_max)) continue;
            IDX2(visited, i, j, fx) = 1;
            if (nreg == cap) {
                cap *= 2;
                accs = (double*)realloc(accs, sizeof(double) * cap);
                merged = (unsigned char*)realloc(merged, cap);
            }
            accs[nreg] = IDX2(d, i, j, fx);
            merged[nreg] = 0;
            nreg += 1;
            IDX2(region, i, j, fx) = (int)nreg;
            int sp = 1;
            memset(in_stack, 0, n);
            if (sk_push_neighbours(i, j, ncx, ncy, fx, stack, &sp, visited, mask, in_stack, d)) { status = 2; break; }
            while (sp - 1 != 0) {
                const int it = stack[2 * (sp - 2)], jt = stack[2 * (sp - 2) + 1];
                sp -= 1;
                if (!IDX2(visited, it, jt, fx)) {
                    accs[nreg - 1] = accs[nreg - 1] + IDX2(d, it, jt, fx);
                    IDX2(visited, it, jt, fx) = 1;
                    if (sk_push_neighbours(it, jt, ncx, ncy, fx, stack, &sp, visited, mask, in_stack, d)) {
                        status = 2;
                        break;
                    }
                    IDX2(region, it, jt, fx) = (int)nreg;
                }
            }
        }
    if (status) goto done;
    {
        int sk = 0;
        for (int i = 1; i <= fx; ++i)
            for (int j = 1; j <= fy; ++j) {
                const int id1 = IDX2(region, i, j, fx);
                if (id1 == 0) continue;
                if (merged[id1 - 1]) continue;
                const double acc = accs[id1 - 1];
                if (fabs(fabs(acc) - particle_number) < skThreshold) {
                    sk += (int)f_nint(copysign(1.0, acc));
                    continue;
                }
                for (int di = -1; di <= 1; ++di)
                    for (int dj = -1; dj <= 1; ++dj) {
                        const int x = (int)f_modulo(i + di - 1, ncx) + 1, y = (int)f_modulo(j + dj - 1, ncy) + 1;
                        if (di == 0 && dj == 0) continue;
                        const int id2 = IDX2(region, x, y, fx);
                        if (id2 == 0) continue;
                        if (merged[id2 - 1]) continue;
                        if (fabs(fabs(accs[id1 - 1] + accs[id2 - 1]) - particle_number) < skThreshold) {
                            merged[id1 - 1] = 1;
                            merged[id2 - 1] = 1;
                        }
                    }
            }
        *out = sk;
    }
done:
    free(mask); free(visited); free(in_stack); free(region); free(stack); free(accs); free(merged);
    return status;
}

/* compute_skyrmion_distribution (rsp:930-983) on a fixed fine density: thresholds
 * max - (i/num)(max - min) outer, sigma = 1 - (s/20)(1 - 1e-5) inner; per pair the counts of
 * particles 1..N, kept when their charge sum rounds closer to nint(total_charge) than the
 * best so far; returns early when the sum is within 0.1 of total_charge. */
int ora_skyrmion_distribution(const double* dens, int fx, int fy, int ncx, int ncy, double total_charge,
                              int N, double min_t, double max_t, int num_thresholds, int* winding)
{
    if (max_t < min_t) return 5;
    int* closest = (int*)calloc(N, sizeof(int));
    double* work = (double*)malloc(sizeof(double) * (size_t)fx * fy);
    if (!closest || !work) { free(closest); free(work); return 4; }
    for (int j = 0; j < N; ++j) winding[j] = 0;
    for (int i = 1; i <= num_thresholds; ++i)
        for (int si = 1; si <= 20; ++si) {
            const double sigma = 1.0 - ((double)si / 20.0) * (1.0 - 0.00001);
            const double thr = max_t - ((double)i / (double)num_thresholds) * (max_t - min_t);
            double w = 0.0;
            long cur = 0;
            for (int j = 1; j <= N; ++j) {
                memcpy(work, dens, sizeof(double) * (size_t)fx * fy);
                int st = ora_skyrmion_number(work, fx, fy, ncx, ncy, thr, j, sigma, &winding[j - 1]);
                if (st) { free(closest); free(work); return st; }
                w = w + (double)(j * winding[j - 1]);
                cur = cur + (long)j * closest[j - 1];
            }
            if (labs(f_nint(w) - f_nint(total_charge)) < labs(cur - f_nint(total_charge)))
                memcpy(closest, winding, sizeof(int) * N);
            if (fabs(w - total_charge) < 0.1) { free(closest); free(work); return 0; }
        }
    memcpy(winding, closest, sizeof(int) * N);
    free(closest); free(work);
    return 0;
}

/* ======================= reference sweep ======================= */
/* UniformRandomInSphere (energyMin.f90:49-68); its pi is the float-rounded literal. */
static void uniform_in_ball(ora_random* rng, double R, double v[3])
{
    double u = 2.0 * ora_uniform(rng) - 1.0;
    double th = acos(u);
    double ph = 2.0 * PI_F * ora_uniform(rng);
    u = ora_uniform(rng);
    double rl = R * pow(u, 1.0 / 3.0);
    v[0] = rl * sin(th) * cos(ph);
    v[1] = rl * sin(th) * sin(ph);
    v[2] = rl * cos(th);
}

static void metropolis_thread(ora_mesh* m, double beta, const ora_params* p, double r,
                              ora_random* rng, long i0, long i1, double* snap,
                              const int* parity)
{
    int N = m->nx, L = m->ny, M = m->nz, stride = 2;
    int iu = N / stride + N % stride, ju = L / stride + L % stride, ku = M / stride + M % stride;
    for (long i = i0; i < i1; ++i) {
        long it = f_nint(ora_uniform(rng) * (iu - 1));
        long jt = f_nint(ora_uniform(rng) * (ju - 1));
        long kt = f_nint(ora_uniform(rng) * (ku - 1));
        it = it * stride + parity[0] % stride; if (it > N - 1) it = N - 1;
        jt = jt * stride + parity[1] % stride; if (jt > L - 1) jt = L - 1;
        kt = kt * stride + parity[2] % stride; if (kt > M - 1) kt = M - 1;
        long cell = cell_index(m, (int)it, (int)jt, (int)kt);
        long ain = 1 + f_nint(ora_uniform(rng) * (m->nsub - 1));
        long at = m->first_atom[cell];
        for (long q = 1; q <= ain - 1; ++q) at = m->next_atom[at];
        double S[3], v[3], Sp[3];
        get_spin(m, at, S);
        uniform_in_ball(rng, r, v);
        for (int d = 0; d < 3; ++d) Sp[d] = S[d] + v[d];
        double n = sqrt(dot3(Sp, Sp));
        for (int d = 0; d < 3; ++d) Sp[d] /= n;
        double oe, ne;
        ora_local_energy(m, at, p, Sp, &oe, &ne);
        double Z = (ne < oe) ? 1.0 : exp(-beta * (ne - oe));
        double pr = ora_uniform(rng);
        if (Z >= pr) {
            snap[at] = Sp[0]; snap[m->natoms + at] = Sp[1]; snap[2 * m->natoms + at] = Sp[2];
        }
    }
}

/* Metropolis_mcs (energyMin.f90:234-374), one thread, demag off. */
void ora_metropolis_mcs_ref(ora_mesh* m, double beta, int n_sweeps, const ora_params* p, double r)
{
    ora_random rng = ora_make_random(0);            /* time*0 + modulo(0,time) = 0, :279-280 */
    for (int i = 0; i < 100; ++i) ora_uniform(&rng); /* :282-284 */
    double* snap = malloc(sizeof(double) * m->natoms * 3);
    for (int sw = 0; sw < n_sweeps; ++sw) {
        int par[3];
        par[0] = 1 + (int)f_nint(ora_uniform(&rng) * (2 - 1));   /* :289-291 */
        par[1] = 1 + (int)f_nint(ora_uniform(&rng) * (2 - 1));
        par[2] = 1 + (int)f_nint(ora_uniform(&rng) * (2 - 1));
        memcpy(snap, m->spins, sizeof(double) * m->natoms * 3);  /* :296-300 */
        metropolis_thread(m, beta, p, r, &rng, 0, m->natoms, snap, par);
        memcpy(m->spins, snap, sizeof(double) * m->natoms * 3);  /* :356-360 */
    }
    free(snap);
}

void ora_metropolis_mcs_omp(ora_mesh* m, double beta, int n_sweeps, const ora_params* p,
                            double r, int n_threads, int time_seed)
{
    if (n_threads < 1) n_threads = 1;
    double* snap = malloc(sizeof(double) * m->natoms * 3);
    ora_random* rngs = malloc(sizeof(ora_random) * n_threads);
    for (int t = 0; t < n_threads; ++t) {
        int tm = time_seed > 0 ? time_seed : 1;
        rngs[t] = ora_make_random((int32_t)(tm * t + t % tm));
        for (int i = 0; i < 100; ++i) ora_uniform(&rngs[t]);
    }
    for (int sw = 0; sw < n_sweeps; ++sw) {
        int par[3];
        par[0] = 1 + (int)f_nint(ora_uniform(&rngs[0]) * (2 - 1));
        par[1] = 1 + (int)f_nint(ora_uniform(&rngs[0]) * (2 - 1));
        par[2] = 1 + (int)f_nint(ora_uniform(&rngs[0]) * (2 - 1));
        memcpy(snap, m->spins, sizeof(double) * m->natoms * 3);
#pragma omp parallel num_threads(n_threads)
        {
            int t = 0, nt = 1;
#ifdef _OPENMP
            t = omp_get_thread_num(); nt = omp_get_num_threads();
#endif
            long chunk = (m->natoms + nt - 1) / nt;           /* static schedule of !$omp do */
            long i0 = t * chunk, i1 = i0 + chunk;
            if (i1 > m->natoms) i1 = m->natoms;
            if (i0 < i1) metropolis_thread(m, beta, p, r, &rngs[t], i0, i1, snap, par);
        }
        memcpy(m->spins, snap, sizeof(double) * m->natoms * 3);
    }
    free(rngs); free(snap);
}

/* ======================= exact colour-class sweep (product keying) ======================= */
static void propose(int move, double r, const double S[3], const double u[4], double Sp[3])
{
    double cz = 2.0 * u[0] - 1.0;
    double st = sqrt((1.0 - cz) * (1.0 + cz));
    double ph = 2.0 * PI_D * (u[1] - 0.5);
    double v[3] = {st * cos(ph), st * sin(ph), cz};
    if (move == 0) { Sp[0] = v[0]; Sp[1] = v[1]; Sp[2] = v[2]; return; }
    double rho = r * cbrt(u[2]);
    for (int d = 0; d < 3; ++d) Sp[d] = S[d] + rho * v[d];
    double n = sqrt(dot3(Sp, Sp));
    for (int d = 0; d < 3; ++d) Sp[d] /= n;
}

static int trial_site(ora_mesh* m, long at, uint32_t sweep, double beta, const ora_params* p,
                      const ora_sweep_key* key, double* de, double* margin)
{
    double u[4], S[3], Sp[3], oe, ne;
    philox_draw(key->seed, (uint32_t)at, sweep, key->replica, key->ensemble, 0,
                key->philox_rounds > 0 ? key->philox_rounds : 10, u);
    get_spin(m, at, S);
    propose(key->move, key->r, S, u, Sp);
    ora_local_energy(m, at, p, Sp, &oe, &ne);
    double dE = ne - oe;
    if (margin) *margin = log(u[3]) + beta * dE;
    int acc = (dE <= 0.0) || (u[3] < exp(-beta * dE));
    if (acc) {
        m->spins[at] = Sp[0]; m->spins[m->natoms + at] = Sp[1]; m->spins[2 * m->natoms + at] = Sp[2];
        *de = dE;
    } else *de = 0.0;
    return acc;
}

long ora_colour_pass(ora_mesh* m, const int* colour_of, int colour, uint32_t sweep,
                     double beta, const ora_params* p, const ora_sweep_key* key,
                     double* de_sum, uint8_t* accepted, double* log_margin)
{
    long nacc = 0;
    double s = 0.0;
    for (long at = 0; at < m->natoms; ++at) {
        if (colour_of[at] != colour) continue;
        double de, mg;
        int a = trial_site(m, at, sweep, beta, p, key, &de, &mg);
        nacc += a;
        s += de;
        if (accepted) accepted[at] = (uint8_t)a;
        if (log_margin) log_margin[at] = mg;
    }
    if (de_sum) *de_sum += s;
    return nacc;
}

long ora_colour_sweeps_omp(ora_mesh* m, const int* colour_of, int n_colours, uint32_t sweep0,
                           int n_sweeps, double beta, const ora_params* p,
                           const ora_sweep_key* key, int n_threads)
{
    long nacc = 0;
    if (n_threads < 1) n_threads = 1;
    for (int sw = 0; sw < n_sweeps; ++sw)
        for (int c = 0; c < n_colours; ++c) {
            long acc = 0;
#pragma omp parallel for num_threads(n_threads) reduction(+:acc) schedule(static)
            for (long at = 0; at < m->natoms; ++at) {
                if (colour_of[at] != c) continue;
                double de;
                acc += trial_site(m, at, sweep0 + (uint32_t)sw, beta, p, key, &de, NULL);
            }
            nacc += acc;
        }
    return nacc;
}

/* ======================= optimised CPU checkerboard (baseline only) ======================= */
/* The fastest CPU form of the sweep, for the CPU baseline: simple cubic, FP32 SoA planes in
 * reference atom order (z fastest), colour (x+y+z)&1, the local-field form of
 * calculateHeisenbergEnergy (energyMin.f90:86-171) with shell-1 exchange, bulk or
 * interfacial DMI about z, Zeeman along z and the -K (S.e)^2 extension, ball or uniform
 * proposals (energyMin.f90:49-68) and Philox4x32-10 draws keyed (site, sweep, replica,
 * ensemble<<8) like the device sweep; OpenMP over (x, y) rows.  Returns accepted trials. */
static inline float cb_u01f(uint32_t x) { return (float)(2u * (x >> 9) + 1u) * (1.0f / 16777216.0f); }

long ora_cb_sweeps_f32(float* sx, float* sy, float* sz, int L, int n_sweeps, uint32_t sweep0,
                       double beta, const ora_params* p, const ora_sweep_key* key, int n_threads)
{
    const int n = L;
    const float J = (float)p->J, D = (float)p->Dz, B = (float)p->B, K = (float)p->K;
    const float ex = (float)p->K_axis[0], ey = (float)p->K_axis[1], ez = (float)p->K_axis[2];
    const float fb = (float)beta, r = (float)key->r;
    const int bulk = p->dmi_bulk, move = key->move;
    const uint32_t k0 = (uint32_t)key->seed, k1 = (uint32_t)(key->seed >> 32);
    const uint32_t cw = (key->ensemble << 8);
    long nacc = 0;
    if (n_threads < 1) n_threads = 1;
    for (int sw = 0; sw < n_sweeps; ++sw)
        for (int colour = 0; colour < 2; ++colour) {
            long acc = 0;
#pragma omp parallel for num_threads(n_threads) reduction(+:acc) schedule(static) collapse(2)
            for (int x = 0; x < n; ++x)
                for (int y = 0; y < n; ++y) {
                    const long row = ((long)x * n + y) * n;
                    const long rxp = ((long)(x + 1 == n ? 0 : x + 1) * n + y) * n;
                    const long rxm = ((long)(x == 0 ? n - 1 : x - 1) * n + y) * n;
                    const long ryp = ((long)x * n + (y + 1 == n ? 0 : y + 1)) * n;
                    const long rym = ((long)x * n + (y == 0 ? n - 1 : y - 1)) * n;
                    for (int z = (x + y + colour) & 1; z < n; z += 2) {
                        const int zp = z + 1 == n ? 0 : z + 1, zm = z == 0 ? n - 1 : z - 1;
                        const long at = row + z;
                        const float pxx = sx[rxp + z], pxy = sy[rxp + z], pxz = sz[rxp + z];
                        const float mxx = sx[rxm + z], mxy = sy[rxm + z], mxz = sz[rxm + z];
                        const float pyx = sx[ryp + z], pyy = sy[ryp + z], pyz = sz[ryp + z];
                        const float myx = sx[rym + z], myy = sy[rym + z], myz = sz[rym + z];
                        const float pzx = sx[row + zp], pzy = sy[row + zp], pzz = sz[row + zp];
                        const float mzx = sx[row + zm], mzy = sy[row + zm], mzz = sz[row + zm];
                        float hx = J * (pxx + mxx + pyx + myx + pzx + mzx);
                        float hy = J * (pxy + mxy + pyy + myy + pzy + mzy);
                        float hz = J * (pxz + mxz + pyz + myz + pzz + mzz);
                        if (bulk) {
                            hx += D * ((mzy - pzy) - (myz - pyz));
                            hy += D * ((mxz - pxz) - (mzx - pzx));
                            hz += D * ((myx - pyx) - (mxy - pxy));
                        } else {
                            hx += D * (pxz - mxz);
                            hy += D * (pyz - myz);
                            hz += D * ((mxx - pxx) - (pyy - myy));
                        }
                        hz -= B;
                        /* Philox4x32-10, counter (site, sweep, replica, ensemble<<8) */
                        uint32_t c0 = (uint32_t)at, c1 = sweep0 + (uint32_t)sw, c2 = key->replica, c3 = cw;
                        uint32_t q0 = k0, q1 = k1;
                        for (int i = 0; i < 10; ++i) {
                            const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
                            c0 = (uint32_t)(p1 >> 32) ^ c1 ^ q0;
                            c1 = (uint32_t)p1;
                            c2 = (uint32_t)(p0 >> 32) ^ c3 ^ q1;
                            c3 = (uint32_t)p0;
                            q0 += 0x9E3779B9u;
                            q1 += 0xBB67AE85u;
                        }
                        const float sxo = sx[at], syo = sy[at], szo = sz[at];
                        const float cz = 2.0f * cb_u01f(c0) - 1.0f;
                        const float st = sqrtf((1.0f - cz) * (1.0f + cz));
                        const float ph = 6.28318531f * (cb_u01f(c1) - 0.5f);
                        float vx = st * cosf(ph), vy = st * sinf(ph), vz = cz;
                        if (move == 1) {
                            const float rho = r * cbrtf(cb_u01f(c2));
                            vx = sxo + rho * vx; vy = syo + rho * vy; vz = szo + rho * vz;
                            const float in = 1.0f / sqrtf(vx * vx + vy * vy + vz * vz);
                            vx *= in; vy *= in; vz *= in;
                        }
                        float dE = (vx - sxo) * hx + (vy - syo) * hy + (vz - szo) * hz;
                        if (K != 0.0f) {
                            const float e1 = vx * ex + vy * ey + vz * ez, e0 = sxo * ex + syo * ey + szo * ez;
                            dE -= K * (e1 * e1 - e0 * e0);
                        }
                        if (dE <= 0.0f || cb_u01f(c3) < expf(-fb * dE)) {
                            sx[at] = vx; sy[at] = vy; sz[at] = vz;
                            ++acc;
                        }
                    }
                }
            nacc += acc;
        }
    return nacc;
}

void ora_init_uniform(ora_mesh* m, uint64_t seed, uint32_t ensemble, uint32_t replica)
{
    for (long at = 0; at < m->natoms; ++at) {
        double u[4];
        philox_draw(seed, (uint32_t)at, 0u, replica, ensemble, 1, 10, u);
        double cz = 2.0 * u[0] - 1.0;
        double st = sqrt((1.0 - cz) * (1.0 + cz));
        double ph = 2.0 * PI_D * (u[1] - 0.5);
        m->spins[at] = st * cos(ph);
        m->spins[m->natoms + at] = st * sin(ph);
        m->spins[2 * m->natoms + at] = cz;
    }
}

/* ======================= stereographic skyrmion ======================= */
/* NSphereProjection (StereographicProjection.f90:58-117) for a 3-vector: returns
 * theta = angles(1), phi = angles(2). */
static void nsphere_projection(const double coord[3], const double centre[3], double R,
                               double* theta, double* phi)
{
    double q[3] = {coord[0] - centre[0], coord[1] - centre[1], 0.0};
    double k = (q[0] * q[0] + q[1] * q[1]) / (4.0 * (R * R));
    double a = k + 1.0, b = -(4.0 * k + 2.0) * R, c = 4.0 * R * R * k;
    double q2 = (-b - sqrt(b * b - 4.0 * a * c)) / (2.0 * a);
    double tp[3];
    tp[0] = (q[0] / (2.0 * R)) * (2.0 * R - q2);
    tp[1] = (q[1] / (2.0 * R)) * (2.0 * R - q2);
    tp[2] = q2 - R;
    double ph = atan2(tp[1], tp[0]);
    if (ph < 0.0) ph = ph + 2.0 * PI_F;   /* 2*3.14159265358979323846 default-real literal, :106 */
    double r = sqrt(tp[0] * tp[0] + tp[1] * tp[1]);
    double th = atan2(r, tp[2]);
    if (th != th || ph != ph) { th = 0.0; ph = 0.0; }
    *theta = th; *phi = ph;
}

/* initialise_skyrmion_sp (LLG.f90:28-73) */
void ora_init_skyrmion(ora_mesh* m, double rx, double ry, double R_s, double chi, int N)
{
    for (long i = 0; i < m->natoms; ++i) {
        double pos[3] = {(double)m->x[i], (double)m->y[i], (double)m->z[i]};
        double cen[3] = {rx, ry, (double)m->z[i] + R_s};
        double th, ph;
        nsphere_projection(pos, cen, R_s, &th, &ph);
        m->spins[i] = sin(th) * cos(N * (ph + chi));
        m->spins[m->natoms + i] = sin(th) * sin(N * (ph + chi));
        m->spins[2 * m->natoms + i] = cos(th);
    }
}

/* ======================= replica exchange ======================= */
void ora_temperature_ladder(double tmin, double tmax, int n, double* T)
{
    for (int j = 0; j < n; ++j)
        T[j] = (n > 1) ? tmin * pow(tmax / tmin, (double)j / (double)(n - 1)) : tmin;
}

/* PT.f90:235-272 */
void ora_pt_swaps_ref(ora_random* rng, int n, int n_swaps, const double* T,
                      const double* E, int* tm)
{
    for (int s = 0; s < n_swaps; ++s) {
        int i1 = (int)f_nint(ora_uniform(rng) * (n - 1)) + 1;   /* 1-based */
        int i2 = (i1 == 1) ? 2 : (i1 == n ? n - 1 : i1 + 1);
        double E1 = E[tm[i1 - 1]], E2 = E[tm[i2 - 1]];
        double b1 = 1.0 / T[i1 - 1], b2 = 1.0 / T[i2 - 1];
        double Delta = (b2 - b1) * (E1 - E2);
        double u = ora_uniform(rng);
        if (u <= 0.0) u = 1e-10;
        u = log(u);
        if (u < Delta) { int t = tm[i1 - 1]; tm[i1 - 1] = tm[i2 - 1]; tm[i2 - 1] = t; }
    }
}

int ora_pt_exchange(uint64_t seed, uint32_t ensemble, uint32_t round, int n, const double* betas,
                    const double* e_rep, int* t2r, int rounds)
{
    int acc = 0;
    for (int t = (int)(round & 1u); t + 1 < n; t += 2) {
        double u[4];
        philox_draw(seed, (uint32_t)t, round, 0u, ensemble, 2, rounds > 0 ? rounds : 10, u);
        double d = (betas[t] - betas[t + 1]) * (e_rep[t2r[t]] - e_rep[t2r[t + 1]]);
        if (d >= 0.0 || u[0] < exp(d)) {
            int x = t2r[t]; t2r[t] = t2r[t + 1]; t2r[t + 1] = x;
            ++acc;
        }
    }
    return acc;
}

/* ======================= tau_int (Sokal automatic window) ======================= */
double ora_tau_int(const double* x, long n, double cw)
{
    if (n < 4) return 0.5;
    double mean = 0.0;
    for (long i = 0; i < n; ++i) mean += x[i];
    mean /= (double)n;
    double c0 = 0.0;
    for (long i = 0; i < n; ++i) c0 += (x[i] - mean) * (x[i] - mean);
    c0 /= (double)n;
    if (c0 <= 0.0) return 0.5;
    double tau = 0.5;
    for (long t = 1; t < n; ++t) {
        double ct = 0.0;
        for (long i = 0; i + t < n; ++i) ct += (x[i] - mean) * (x[i + t] - mean);
        ct /= (double)n;
        tau += ct / c0;
        if ((double)t >= cw * tau) break;
    }
    return tau;
}

/* ======================= Fortran edit descriptors ======================= */
/* F0.d: minimal width, d decimals; the optional zero before the point is omitted for
 * |x| < 1 (the consumer unified-analysis.py:234-247 strips it to rebuild file names). */
int ora_fmt_F0(char* buf, double x, int d)
{
    if (x != x) return sprintf(buf, "NaN");
    if (isinf(x)) return sprintf(buf, x > 0 ? "Infinity" : "-Infinity");
    char tmp[400];
    snprintf(tmp, sizeof tmp, "%.*f", d, x);
    const char* s = tmp;
    int neg = signbit(x) ? 1 : 0;   /* a negative internal value keeps its minus sign */
    if (*s == '-') ++s;
    if (s[0] == '0' && s[1] == '.') ++s;
    return sprintf(buf, "%s%s", neg ? "-" : "", s);
}

/* Im.m with w = 0: at least m digits */
int ora_fmt_I0m(char* buf, long v, int m)
{
    if (v < 0) return sprintf(buf, "-%0*ld", m, -v);
    return sprintf(buf, "%0*ld", m, v);
}

/* ESw.d: scientific, one non-zero digit before the point, exponent E+dd (or +ddd without
 * the E when |exp| > 99), right-justified in w. */
int ora_fmt_ES(char* buf, double x, int w, int d)
{
    char tmp[128], out[160];
    if (x != x) { snprintf(out, sizeof out, "NaN"); }
    else {
        snprintf(tmp, sizeof tmp, "%.*e", d, x);
        char* e = strchr(tmp, 'e');
        int ex = atoi(e + 1);
        *e = 0;
        if (ex > 99 || ex < -99) snprintf(out, sizeof out, "%s%+04d", tmp, ex);
        else snprintf(out, sizeof out, "%sE%+03d", tmp, ex);
    }
    int n = (int)strlen(out);
    if (n > w) { for (int i = 0; i < w; ++i) buf[i] = '*'; buf[w] = 0; return w; }
    int pad = w - n;
    memset(buf, ' ', pad);
    memcpy(buf + pad, out, n + 1);
    return w;
}

/* E0.d: 0.ddddE<sign><digits> with the mantissa in [0.1,1) and the exponent written with
 * no leading zeros (the form unified-analysis.py:178-199 rebuilds). */
int ora_fmt_E0(char* buf, double x, int d)
{
    if (x == 0.0) return sprintf(buf, "0.%0*dE+0", d, 0);
    char tmp[128];
    snprintf(tmp, sizeof tmp, "%.*e", d - 1, fabs(x));
    char* e = strchr(tmp, 'e');
    int ex = atoi(e + 1) + 1;
    *e = 0;
    /* tmp = "D.ddd" -> "0.Dddd" */
    char mant[128];
    int k = 0;
    mant[k++] = '0'; mant[k++] = '.'; mant[k++] = tmp[0];
    for (const char* q = tmp + 2; *q; ++q) mant[k++] = *q;
    mant[k] = 0;
    return sprintf(buf, "%s%sE%+d", x < 0 ? "-" : "", mant, ex);
}
