/*
 * ising_oracle.h -- CPU FP64 restatement of the reference's Heisenberg Monte Carlo path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA product in
 * ising_b200/; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline /
 * reference arm may load it.  The product never links, imports or falls back to it.
 *
 * Parity status: the reference (SamuelJosephs/ISING, Fortran 2008) ships no golden
 * vectors, known-answer tests or fixtures for this path, and it cannot be built in this
 * image (no gfortran, MPI or FFTW).  Parity is therefore UNPINNED by the reference; this
 * restatement is pinned by analytic known answers (uniform states, the stereographic
 * skyrmion of src/LLG.f90:28-73 giving Q = +-1) and by committed fixtures it generates.
 *
 * Every routine cites the reference file:line it restates.  Indices are 0-based here;
 * the reference is 1-based (atom i here is atom i+1 there).
 */
#ifndef ISING_ORACLE_H
#define ISING_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- constants (src/constants.f90:9-16) ---------------- */
/* The reference writes these as default-real (single precision) literals assigned to
 * real(8) parameters, so their values are the float-rounded ones; kept that way here. */
double ora_const_kb(void);      /* 8.6173303e-5 rounded to float  */
double ora_const_pi_f(void);    /* 3.14159265358979323846 rounded to float */
double ora_const_g(void);       /* 2.0 */
double ora_const_mu_b(void);    /* 1.0 */

/* ---------------- reference RNG (src/rand.f90:11-95) ---------------- */
typedef struct { int32_t seed, ix, iy; } ora_random;
ora_random ora_make_random(int32_t seed);
double ora_uniform(ora_random* r);
/* fill out[n] with successive draws of makeRandom(seed) (for tests) */
void ora_uniform_stream(int32_t seed, int n, double* out);

/* ---------------- Philox4x32-10 (Salmon et al., SC'11) ---------------- */
void ora_philox4x32(const uint32_t ctr[4], const uint32_t key[2], int rounds, uint32_t out[4]);
/* (0,1) uniform from 23 high bits: (2*(x>>9)+1) * 2^-24, exact in float and double */
double ora_u01(uint32_t x);

/* ---------------- lattice (src/chainMesh.f90:729-911) ---------------- */
typedef struct ora_mesh ora_mesh;

/* frac_xyz: n_sub x 3 fractional coordinates (real(4) in the reference, Atom_t%x).
 * shell_tol <= 0 -> 0.1*a (chainMesh.f90:783); n_shells <= 0 -> 2 (:784). */
ora_mesh* ora_mesh_create(const float* frac_xyz, int n_sub, int nx, int ny, int nz,
                          double a, double b, double c,
                          double ab_deg, double bc_deg, double ca_deg,
                          double shell_tol, int n_shells);
void ora_mesh_destroy(ora_mesh* m);
long ora_mesh_natoms(const ora_mesh* m);
void ora_mesh_vectors(const ora_mesh* m, double out[18]); /* a,b,c then ar,br,cr */
void ora_mesh_positions(const ora_mesh* m, float* xyz /* natoms x 3 row-major */);
int  ora_mesh_first_atom(const ora_mesh* m, long cell);
/* shells: number of entries of atom i in shell s, and copy of the list (0-based) */
int  ora_mesh_shell_size(const ora_mesh* m, long atom, int shell);
int  ora_mesh_shell_list(const ora_mesh* m, long atom, int shell, int* out);
int  ora_mesh_nl_size(const ora_mesh* m, long atom);
int  ora_mesh_nl_list(const ora_mesh* m, long atom, int* out);
/* derivativeList(atom, d, lo/hi) -> 0-based atom; d in 0..2, side 0 = lower, 1 = higher */
int  ora_mesh_deriv(const ora_mesh* m, long atom, int d, int side);
/* spins: atomSpins(numAtoms,3) column-major, FP64 */
double* ora_mesh_spins(ora_mesh* m);
/* minimum-image vector r_j - r_i (distance_points_vec, chainMesh.f90:206-241) */
void ora_mesh_min_image(const ora_mesh* m, long i, long j, double out[3]);

/* ---------------- energies (src/energyMin.f90) ---------------- */
typedef struct {
    double J, J_prime, Dz, Dz_prime, B;
    double K;            /* extension: -K (S.e)^2, no reference counterpart */
    double K_axis[3];
    int    dmi_bulk;     /* 0: reference D = Dz c_hat x r_hat (:114,137); 1: D = Dz r_hat (:138) */
} ora_params;

/* calculateHeisenbergEnergy (src/energyMin.f90:86-171), demag off. */
void ora_local_energy(const ora_mesh* m, long atom, const ora_params* p,
                      const double s_prop[3], double* old_e, double* new_e);
/* TotalHeisenbergEnergy (src/energyMin.f90:499-528 with helper :174-229), demag off.
 * zeeman_gmu: the reference uses g*mu_B = 2 (:222).  anisotropy adds -K (S.e)^2 per site. */
double ora_total_energy(const ora_mesh* m, const ora_params* p, double zeeman_gmu);
/* The same Hamiltonian as the local routine, summed once per site and bond:
 * sum_<ij> [J S.S + D.(SxS)] + J' sum_<<ij>> S.S - B sum S_z - K sum (S.e)^2  (shell lists) */
double ora_canonical_energy(const ora_mesh* m, const ora_params* p);

/* ---------------- winding number (reciprocalSpaceProcesses.f90:284-364) ---------------- */
double ora_arc_winding(const double s1[3], const double s2[3], const double s3[3]);
double ora_winding_number(const ora_mesh* m, int z_1based);
void   ora_winding_density(const ora_mesh* m, int z_1based, double* dens /* nx*ny col-major */);
/* ---------------- skyrmion counting (reciprocalSpaceProcesses.f90:582-983) ---------------- */
void ora_gaussian_kernel(double sigma, double G[25]);
int ora_gaussian_filter_2d(double* a, int nx, int ny, double sigma);
int ora_skyrmion_number(double* dens, int fx, int fy, int ncx, int ncy, double q_threshold,
                        int particle_number, double sigma, int* out);
int ora_skyrmion_distribution(const double* dens, int fx, int fy, int ncx, int ncy, double total_charge,
                              int N, double min_t, double max_t, int num_thresholds, int* winding);
/* chainMesh_statistics (src/PT-Utils.f90:33-66) without the skyrmion count */
void   ora_statistics(const ora_mesh* m, double* wnd_mid, double* wnd_spread, double mag[3]);

/* ---------------- sweeps ---------------- */
/* Metropolis_mcs (src/energyMin.f90:234-374) restated for one thread, demag off:
 * seed = time*0 + mod(0,time) = 0 for thread 0 (:279-280), 100 warm-up draws (:282-284),
 * random parity cell per trial (:307-321), ball proposal (:323-329), snapshot (Jacobi)
 * semantics (:296-300,356-360).  Deterministic. */
void ora_metropolis_mcs_ref(ora_mesh* m, double beta, int n_sweeps, const ora_params* p,
                            double r);
/* Same algorithm with n_threads OpenMP threads, thread t seeded like the reference
 * (makeRandom(time*t + mod(t,time)), time given).  Used as the timed CPU reference arm. */
void ora_metropolis_mcs_omp(ora_mesh* m, double beta, int n_sweeps, const ora_params* p,
                            double r, int n_threads, int time_seed);

/* Exact colour-class Metropolis sweep with the product's Philox keying, in FP64.
 * colour_of[atom] gives the class; classes are swept 0..n_colours-1 in order.
 * move: 0 = fresh uniform unit vector, 1 = ball step of radius r (energyMin.f90:49-68).
 * Returns the accepted count; accumulates dE into *de_sum. */
typedef struct {
    uint64_t seed;
    uint32_t ensemble, replica;
    int move;
    double r;
    int philox_rounds;
} ora_sweep_key;
/* Optimised FP32 checkerboard sweep of a simple cubic L^3 mesh (CPU baseline only): SoA planes
 * in reference atom order, OpenMP over rows; returns accepted trials. */
long ora_cb_sweeps_f32(float* sx, float* sy, float* sz, int L, int n_sweeps, uint32_t sweep0,
                       double beta, const ora_params* p, const ora_sweep_key* key, int n_threads);
long ora_colour_pass(ora_mesh* m, const int* colour_of, int colour, uint32_t sweep,
                     double beta, const ora_params* p, const ora_sweep_key* key,
                     double* de_sum, uint8_t* accepted /* natoms or NULL */,
                     double* log_margin /* natoms or NULL: ln(u) + beta*dE */);
/* Checkerboard sweeps over an SC/any mesh with an explicit colouring, OpenMP over sites
 * of one class (the conservative CPU baseline).  Returns accepted count. */
long ora_colour_sweeps_omp(ora_mesh* m, const int* colour_of, int n_colours,
                           uint32_t sweep0, int n_sweeps, double beta, const ora_params* p,
                           const ora_sweep_key* key, int n_threads);

/* uniform unit vectors from Philox(seed; site, 0, replica, ensemble|tag) */
void ora_init_uniform(ora_mesh* m, uint64_t seed, uint32_t ensemble, uint32_t replica);

/* Stereographic skyrmion (src/LLG.f90:28-73 with NSphereProjection,
 * src/StereographicProjection.f90:58-117). centre = (rx, ry, *). */
void ora_init_skyrmion(ora_mesh* m, double rx, double ry, double R_s, double chi, int N);

/* ---------------- replica exchange (src/PT.f90:199-272) ---------------- */
/* geometric ladder T_j = Tmin (Tmax/Tmin)^(j/(n-1)), j = 0..n-1 (PT.f90:202) */
void ora_temperature_ladder(double tmin, double tmax, int n, double* T);
/* Reference swap block restated (PT.f90:235-272): n_swaps attempts; Index1 =
 * nint(u*(n-1))+1; partner; Delta = (b2-b1)(E1-E2) with b = 1/T (no k_B); accept if
 * log(u) < Delta.  energies[] indexed by replica (mesh index), temp_mesh[j] = mesh at
 * temperature j (0-based).  Consumes draws from rng. */
void ora_pt_swaps_ref(ora_random* rng, int n_temps, int n_swaps, const double* T,
                      const double* energies, int* temp_mesh);
/* Correct criterion, deterministic even/odd neighbour pairs keyed by Philox
 * (seed; pair, round, ensemble, tag 2): accept if u < exp((b_i - b_j)(E_i - E_j)).
 * betas[t] per temperature slot. Returns accepted count; updates temp_to_rep. */
int ora_pt_exchange(uint64_t seed, uint32_t ensemble, uint32_t round, int n_temps,
                    const double* betas, const double* e_rep, int* temp_to_rep,
                    int philox_rounds);

/* ---------------- statistics helpers ---------------- */
/* Sokal automatic-window integrated autocorrelation time (c = 5). */
double ora_tau_int(const double* x, long n, double c_window);

/* ---------------- Fortran edit descriptors used by the CSV outputs ---------------- */
/* gfortran F0.d (no leading zero for |x|<1), I0.m, ESw.d, E0.d; return length */
int ora_fmt_F0(char* buf, double x, int d);
int ora_fmt_I0m(char* buf, long v, int m);
int ora_fmt_ES(char* buf, double x, int w, int d);
int ora_fmt_E0(char* buf, double x, int d);

#ifdef __cplusplus
}
#endif
#endif
