/*
 * ising_gpu.h -- C-ABI of libisinggpu.so, the B200 (sm_100a) Heisenberg Monte Carlo path.
 *
 * Drop-in boundary for the Fortran drivers of SamuelJosephs/ISING (src/PT.f90,
 * src/ISING.f90).  Every entry point replaces one reference routine or inline block;
 * the replaced interface is cited beside each declaration (paths within the reference
 * project).  A Fortran `bind(C)` module over these symbols lets the drivers switch by
 * changing `use` lines.
 *
 * Conventions
 *  - Plain C types only; no CUDA or framework types cross this boundary.
 *  - Every call returns an int status (ISING_OK = 0) and never aborts; on failure
 *    ising_last_error() gives a message (thread-local).
 *  - Host spin arrays are FP64 column-major (numAtoms, 3), the layout of
 *    ChainMesh_t%atomSpins (src/chainMesh.f90:20).  Atom order is the reference's:
 *    atom = cell*n_sub + i, cell = (ix*ny + iy)*nz + iz (src/chainMesh.f90:684,878).
 *  - Indices at this boundary are 0-based unless a name ends in _1based.
 *  - The library owns device memory (FP32 SoA spins, FP64 accumulators, lattice tables)
 *    behind opaque handles; one CUDA stream per handle; one host thread per handle.
 *  - Energy sign convention is the reference's: E = +J S_i.S_j (src/energyMin.f90:139),
 *    so a ferromagnet has J < 0.
 */
#ifndef ISING_GPU_H
#define ISING_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status codes */
#define ISING_OK 0
#define ISING_ERR_ARG 1          /* bad argument (the reference calls error stop / MPI_Abort) */
#define ISING_ERR_NAN 2          /* NaN in spins or proposals (src/energyMin.f90:330-331) */
#define ISING_ERR_BOUNDS 3       /* index out of range (e.g. Z_index, rsp:334) */
#define ISING_ERR_TIMEOUT 4      /* a bounded device-side wait gave up */
#define ISING_ERR_UNSUPPORTED 5  /* e.g. demag=.true. in parallel tempering */
#define ISING_ERR_CUDA 6         /* CUDA runtime error or no usable device */
#define ISING_ERR_ALLOC 7        /* device or host allocation failed */
#define ISING_ERR_LATTICE 8      /* derivative list incomplete ("Unable to locate atoms",
                                    src/chainMesh.f90:1028) */
#define ISING_ERR_CAPACITY 9     /* region-growth stack of 10000 rows full ("Stack array
                                    capacity exceeded", rsp:611) */

const char* ising_status_string(int status);
const char* ising_last_error(void);
/* Library version, e.g. "isinggpu 0.1 sm_100a". */
const char* ising_version(void);

/* ---------------------------------------------------------------- unit cells */
#define ISING_CELL_SC 0            /* simple cubic, one atom at the origin (no reference cell) */
#define ISING_CELL_BCC 1           /* bcc_unit_cell, src/unit_cells.f90:7-30 */
#define ISING_CELL_HYPER_KAGOME 2  /* hyper_kagome_unit_cell, src/unit_cells.f90:32-77 */

/* Fills the Bravais parameters and fractional atom coordinates of a unit cell.
 * frac_xyz receives n_atoms x 3 floats (row-major), at most 12 atoms.
 * Replaces bcc_unit_cell / hyper_kagome_unit_cell (src/unit_cells.f90:7,32). */
int ising_unit_cell(int kind, double* a, double* b, double* c, double* ab_deg,
                    double* bc_deg, double* ca_deg, float* frac_xyz, int* n_atoms);

/* ---------------------------------------------------------------- lattice + state */
typedef struct ising_mesh ising_mesh;

typedef struct {
    int64_t num_atoms;       /* ChainMesh_t%numAtoms */
    int64_t num_cells;       /* ChainMesh_t%numChainMeshCells */
    int nx, ny, nz, n_sub;   /* numCellsX/Y/Z, atoms per unit cell */
    int n_shells;            /* neighbour shells built (default 2) */
    int n_replicas;          /* replica spin buffers held on the device */
    int shell_size[2];       /* entries per atom in shells 1 and 2 (sublattice 0) */
    int checkerboard;        /* storage order of the spins on the device: 1 the SC 2-colour fast path
                                (even nx, ny; nz % 4 == 0); 2 the octant order of other crystals
                                with even extents (blocks of cells/8 sites per cell octant
                                and sublattice; each colour class is a set of blocks); 3
                                sublattice planes of
                                two-sublattice crystals whose first shell joins only the two
                                sublattices (BCC; the colour classes are the sublattices);
                                0 the reference atom order */
    double a_vec[3], b_vec[3], c_vec[3];
} ising_mesh_info;

/* Builds the lattice and allocates n_replicas spin buffers on `device`.
 * Replaces makeChainMesh(numCellsX, numCellsY, numCellsZ, AtomsInUnitCell, a, b, c,
 * ab_deg, bc_deg, ca_deg [, distance_threshold, numShells]) (src/chainMesh.f90:729-732).
 * shell_tol <= 0 selects 0.1*a (:783); n_shells <= 0 selects 2 (:784).
 * Requires nx, ny, nz >= 3 (smaller meshes stop the reference at :1028).
 * device = -1 builds the lattice tables only (no GPU state); calls that need spins then
 * return ISING_ERR_ARG. */
int ising_mesh_create(const float* frac_xyz, int n_atoms_cell, int nx, int ny, int nz,
                      double a, double b, double c, double ab_deg, double bc_deg,
                      double ca_deg, double shell_tol, int n_shells, int n_replicas,
                      int device, ising_mesh** out);
/* Replaces deallocateChainMesh (src/chainMesh.f90:914-929). */
int ising_mesh_destroy(ising_mesh* mesh);
int ising_mesh_get_info(const ising_mesh* mesh, ising_mesh_info* info);
/* Issue the handle's device work on an external CUDA stream (a cudaStream_t passed as an
 * opaque pointer); NULL restores the handle's own stream.  No reference counterpart. */
int ising_mesh_set_stream(ising_mesh* mesh, void* cuda_stream);
/* Atom positions, real(4) like Atom_t%x,y,z (src/atom.f90:5): xyz is num_atoms x 3 row-major. */
int ising_mesh_positions(const ising_mesh* mesh, float* xyz);
/* Neighbour list of one atom, expanded from the lattice tables:
 * shell 0/1 = atomShells(atom, 1/2)%NNList (src/chainMesh.f90:41,495-591);
 * shell -1 = the legacy atoms(atom)%NeighborList (src/atom.f90:9, chainMesh.f90:280-405).
 * Writes up to cap entries, returns the count in *n. */
int ising_mesh_neighbours(const ising_mesh* mesh, int64_t atom, int shell, int64_t* out,
                          int cap, int* n);
/* derivativeList(atom, d, side) (src/chainMesh.f90:23,931-1031), 0-based atoms,
 * out is num_atoms x 3 x 2 row-major (side 0 = lower, 1 = higher). */
int ising_mesh_derivative_list(const ising_mesh* mesh, int64_t* out);

/* Spins of one replica from / to a host FP64 column-major (num_atoms, 3) array
 * (ChainMesh_t%atomSpins, src/chainMesh.f90:20).  set rejects NaN or zero vectors. */
int ising_spins_set(ising_mesh* mesh, int replica, const double* col_major_n3);
int ising_spins_get(const ising_mesh* mesh, int replica, double* col_major_n3);
/* Asynchronous forms (no reference counterpart): queue the transfer of one replica and return.
 * Downloads and uploads run on two streams of their own, after the work already issued on the
 * mesh, so opposite directions overlap; an upload of replica r waits for the last download of
 * r (and vice versa), so one host array can be read back and sent again without a host wait.
 * The host array must stay valid, and unmodified by the host, until ising_spins_wait returns;
 * use pinned memory for overlap.  ising_spins_wait waits for every queued transfer and reports
 * invalid uploaded spins (ISING_ERR_NAN); every other call on the mesh, or on a PT object or
 * engine using it, waits for them first.  The first queued transfer of a replica allocates a
 * device staging buffer of 24 bytes per site for it, kept until the mesh is destroyed. */
int ising_spins_get_async(ising_mesh* mesh, int replica, double* col_major_n3);
int ising_spins_set_async(ising_mesh* mesh, int replica, const double* col_major_n3);
int ising_spins_wait(ising_mesh* mesh);
/* Uniform unit vectors on every replica from Philox(seed; site, 0, replica, ensemble|1).
 * The reference leaves PT spins uninitialised (src/chainMesh.f90:889-890). */
int ising_spins_init_uniform(ising_mesh* mesh, uint64_t seed, uint32_t ensemble);

/* ---------------------------------------------------------------- Hamiltonian */
#define ISING_DMI_INTERFACIAL 0   /* D_ij = Dz * n x r_ij, n = dmi_axis (src/energyMin.f90:114,137) */
#define ISING_DMI_BULK 1          /* D_ij = Dz * r_ij, the commented form (src/energyMin.f90:138) */

typedef struct {
    /* the reference's argument list (src/energyMin.f90:86-87, 234-235, 499) */
    double J, J_prime, Dz, Dz_prime, B;
    /* uniaxial anisotropy -K (S.e)^2: an extension with no reference counterpart */
    double K;
    double K_axis[3];
    /* Zeeman prefactor: 1 in calculateHeisenbergEnergy (:161), g*mu_B = 2 in
     * TotalHeisenbergEnergy (:222, src/constants.f90:11,14) */
    double zeeman_factor;
    int include_Jp;      /* 1: add the J' shell-2 sum (local routine); 0: total routine */
    int dmi_mode;        /* ISING_DMI_INTERFACIAL or ISING_DMI_BULK */
    double dmi_axis[3];  /* interfacial axis; all zero selects c_vec/|c_vec| (:114) */
    int legacy_neighbours; /* 1: sum over the legacy NeighborList (TotalHeisenbergEnergy) */
    int demag;           /* 1: the demagnetising field enters as -mu_0 S.H in the local energy and
                            the sweeps, -1/2 mu_0 S.H in the total energy (mu_0 of
                            src/constants.f90:15); parallel tempering and the batched engine
                            return ISING_ERR_UNSUPPORTED for it (the reference's drivers run with
                            demag = .false., src/PT.f90:29, src/ISING.f90:46) */
} ising_params;

/* Fills p with the conventions of one reference routine:
 * which = 0: calculateHeisenbergEnergy / Metropolis_mcs (zeeman 1, J' on, axis c_hat)
 * which = 1: TotalHeisenbergEnergy (zeeman g*mu_B = 2, J' off, axis z, legacy list). */
int ising_params_reference(int which, double J, double J_prime, double Dz, double Dz_prime,
                           double B, ising_params* p);

/* Colour class of every atom as the sweep uses it for the Hamiltonian p: the checkerboard
 * (x+y+z)&1 on simple-cubic meshes with even nx, ny, nz % 4 == 0 and no J'; the sublattice on
 * BCC meshes (layout 3) without J'; on other crystals
 * with even extents whose shells 1-2 never join one sublattice at an all-even non-zero cell
 * offset (BCC and hyper-kagome, src/unit_cells.f90:7-77), classes of whole blocks (cell octant
 * (x&1, y&1, z&1), sublattice) with no bond of the active shells among them: the fewer of the
 * octant x sublattice-group classes (without J', where shell 1 joins no sublattice to itself,
 * the fewest sublattice sets free of shell-1 bonds at any offset, every octant of each: 3 on
 * hyper-kagome) and a DSatur colouring of the blocks (15 on hyper-kagome with J'); a verified
 * greedy colouring of the active shells otherwise.  No reference counterpart: Metropolis_mcs
 * draws random parity cells instead (src/energyMin.f90:288-316). */
int ising_mesh_colouring(ising_mesh* mesh, const ising_params* p, int* colour_of, int* n_colours);

/* ---------------------------------------------------------------- energies */
/* Replaces calculateHeisenbergEnergy(chainMesh, atomIndex, J, J', Dz, Dz', B, lockArray,
 * S_proposed, oldEnergy, newEnergy, demag_array, demag) (src/energyMin.f90:86-171).
 * FP32 local field on the device, results widened to FP64. */
int ising_local_energy(const ising_mesh* mesh, int replica, int atom_index_1based,
                       const ising_params* p, const double s_prop[3], double* old_e,
                       double* new_e);
/* Batched form of the above for n sites (0-based), s_prop n x 3 row-major. */
int ising_local_energy_batch(const ising_mesh* mesh, int replica, int n, const int64_t* atoms,
                             const double* s_prop, const ising_params* p, double* old_e,
                             double* new_e);
/* Replaces TotalHeisenbergEnergy(chainMesh, J, J', Dz, Dz', B, lockArray, totalEnergy,
 * demag) (src/energyMin.f90:499-528): FP32 terms, FP64 block sums. */
int ising_total_energy(const ising_mesh* mesh, int replica, const ising_params* p, double* e);
/* Replaces calculate_demagnetisation_field(chainMesh, outputArray)
 * (src/reciprocalSpaceProcesses.f90:202-281): the demagnetising field of one replica's spins at
 * every atom, H[3 * numAtoms] column-major as outputArray(numAtoms, 3), FP64.  Cloud-in-cell
 * deposit onto the cell centres (27 neighbouring cells), forward transform, H(k) = -(k.M/k^2) k
 * with k = 0 and the bins beyond pi/a, pi/b, pi/c removed, backward transform / (N L M), and the
 * same weights back to the atoms.  Metropolis sweeps with demag recompute it at the start and
 * every int(pi sqrt(5) / (2 r)) sweeps (src/energyMin.f90:258-259, 363-366). */
int ising_demag_field(const ising_mesh* mesh, int replica, double* H);
/* Replaces write_demagnetisation_field_to_file(chainMesh, demag_field, filepath)
 * (src/energyMin.f90:559-583) for the field of one replica's current spins: header
 * x,y,z,fx,fy,fz, one record per atom, every value F8.4. */
int ising_write_demag_csv(const ising_mesh* mesh, int replica, const char* path);
/* Same result as ising_total_energy, but allocates no device memory: the per-block partial
 * sums live in a fixed array inside the library (128 KiB per device, held until exit), so
 * callers that cannot call cudaMalloc -- loops that must not stall other streams, work
 * issued while another thread captures a graph, applications that reserve device memory up
 * front -- can still evaluate energies.  Replicas are limited to 16,777,216 atoms (larger
 * ones return ISING_ERR_ARG).  All calls on a device share that array: calls that overlap
 * on the GPU race, so issue them one after another.  The first call on a device looks up
 * the array's address; make it before any stream capture.  The address is kept until the
 * process exits, so do not call this again on a device after cudaDeviceReset on it.  No
 * counterpart in the reference. */
int ising_total_energy_noalloc(const ising_mesh* mesh, int replica, const ising_params* p, double* e);
/* Energy and magnetisation vector of every replica in one pass: e[R], m[R*3]. */
int ising_observables(const ising_mesh* mesh, const ising_params* p, double* e, double* m);

/* ---------------------------------------------------------------- sweeps */
#define ISING_MOVE_UNIFORM 0   /* fresh uniform unit vector */
#define ISING_MOVE_BALL 1      /* S' = norm(S + r*ball), UniformRandomInSphere (src/energyMin.f90:49-68) */

/* Replaces Metropolis_mcs(chainMesh, beta, numMCSSweeps, J, J', Dz, Dz', B, r, lockArray,
 * demag) (src/energyMin.f90:234-374).  A sweep visits every atom once through colour
 * classes (checkerboard on even simple-cubic meshes, the two sublattices on BCC meshes
 * without J', octant classes on other crystals with even extents, greedy colouring
 * otherwise) with
 * Philox keyed by (seed, ensemble 0, replica, sweep, atom); the per-replica sweep counter
 * lives in the handle so successive calls continue the stream.  r > 0 selects the ball
 * move of radius r, r <= 0 the uniform move.  lockArray has no counterpart (no locks). */
int ising_metropolis_mcs(ising_mesh* mesh, int replica, double beta, int n_sweeps,
                         const ising_params* p, double r, uint64_t seed);

/* ---------------------------------------------------------------- winding number */
/* Replaces calculate_winding_number2(chainMesh, Z_index) (rsp:320-364). FP64 on device. */
int ising_winding_number(const ising_mesh* mesh, int replica, int z_1based, double* q);
/* All nz slices of one replica (the loop of src/PT-Utils.f90:49-51). */
int ising_winding_all_slices(const ising_mesh* mesh, int replica, double* q_per_slice);
/* Replaces chainMesh_statistics (src/PT-Utils.f90:33-66) except the skyrmion count. */
int ising_statistics(const ising_mesh* mesh, int replica, double* wnd_mid, double* wnd_spread,
                     double m[3]);
/* Replaces calculate_winding_number_density (rsp:438-500): nx x ny column-major, computed
 * by the winding kernel in FP64 on the device. */
int ising_winding_density(const ising_mesh* mesh, int replica, int z_1based, double* density);
/* The densities of all nz slices in one launch and one download: nz consecutive nx x ny
 * column-major slices (the loop of write_winding_number_density, rsp:560-571). */
int ising_winding_density_all(const ising_mesh* mesh, int replica, double* density);

/* ---------------------------------------------------------------- skyrmion counting */
/* Fine-grid scale factors of makeChainMesh's sclx, scly (src/chainMesh.f90:745-773; default
 * 10, each >= 2 or ISING_ERR_ARG). */
int ising_mesh_set_interpolation_scale(ising_mesh* mesh, int sclx, int scly);
int ising_mesh_interpolation_scale(const ising_mesh* mesh, int* sclx, int* scly);
/* Replaces calculate_winding_density_interpolated (rsp:366-436): (sclx*nx) x (scly*ny)
 * column-major density of slice z on the band-limited interpolation of the slice's
 * first-atom spins (the reference's FFTW layout is not reproducible; see DESIGN). */
int ising_winding_density_interpolated(const ising_mesh* mesh, int replica, int z_1based,
                                       double* density);
/* Replaces calculate_skyrmion_number(chainMesh, Z_index, q_threshold, particle_number,
 * sigma) (rsp:627-812).  ISING_ERR_CAPACITY where the reference stops on a full stack. */
int ising_skyrmion_number(const ising_mesh* mesh, int replica, int z_1based, double q_threshold,
                          int particle_number, double sigma, int* skyrmion_number);
/* Replaces compute_skyrmion_distribution(chainMesh, N, winding_array, min_threshold,
 * max_threshold, num_thresholds, Z_index) (rsp:930-983): winding_array[N]. */
int ising_skyrmion_distribution(const ising_mesh* mesh, int replica, int N, double min_threshold,
                                double max_threshold, int num_thresholds, int z_1based,
                                int* winding_array);
/* Replaces chainMesh_statistics (src/PT-Utils.f90:33-66) including skyrmion_number_middle. */
int ising_chain_mesh_statistics(const ising_mesh* mesh, int replica, int* skyrmion_number_middle,
                                double* wnd_mid, double* wnd_spread, double m[3]);
/* Replaces Gaussian_filter_2d(array, sigma) (rsp:814-859) on a host nx x ny column-major
 * array (nx, ny >= 5), computed on the current device. */
int ising_gaussian_filter_2d(double* array, int nx, int ny, double sigma);
/* calculate_skyrmion_number after its interpolation step, on a caller-supplied fx x fy fine
 * density; nx, ny are the coarse cell counts the reference wraps with. */
int ising_skyrmion_number_density(const double* density, int fx, int fy, int nx, int ny,
                                  double q_threshold, int particle_number, double sigma,
                                  int* skyrmion_number);

/* ---------------------------------------------------------------- parallel tempering */
typedef struct ising_pt ising_pt;

#define ISING_PT_EVEN_ODD 0     /* deterministic alternating neighbour pairs, correct criterion */
#define ISING_PT_RANDOM_PAIRS 1 /* n random neighbour pairs per round (src/PT.f90:236-244),
                                   correct criterion */

typedef struct {
    uint64_t seed;
    uint32_t ensemble;        /* Philox key component; distinct per ensemble */
    int move;                 /* ISING_MOVE_UNIFORM or ISING_MOVE_BALL */
    double r;                 /* ball radius (src/PT.f90:230 uses 0.2) */
    int scheme;               /* ISING_PT_EVEN_ODD or ISING_PT_RANDOM_PAIRS */
    int resync_every;         /* rounds between FP64 energy resyncs (0 = never) */
    int record;               /* 1: record E, |M|, Q per sweep into a device series */
    int record_capacity;      /* sweeps to keep per replica when record = 1 */
    int l2_group;             /* replicas per group of the L2-paired sweep schedule, or of the
                                 octant schedule (every sweep of a group, then the next; 0 = auto) */
    int sweep_kernel;         /* checkerboard meshes: 0 auto, 1 register kernel, 2 TMA-staged kernel;
                                 octant meshes: 0 or 1 one launch per colour class, 3 one
                                 persistent launch per round (bit-identical) */
} ising_pt_options;

/* Replaces the PT state of src/PT.f90:193-204 (TemperatureMeshArray, TemperatureArray):
 * replicas 0..n_temps-1 of `mesh` start at temperature slots 0..n_temps-1 with inverse
 * temperatures betas[t]. */
int ising_pt_create(ising_mesh* mesh, int n_temps, const double* betas, const ising_params* p,
                    const ising_pt_options* opt, ising_pt** out);
/* destroy a PT object before its mesh */
int ising_pt_destroy(ising_pt* pt);
/* rounds x [sweeps_per_swap sweeps of every replica, then one exchange], replacing the
 * iteration loop of src/PT.f90:219-273; replayed from a CUDA graph. */
int ising_pt_run(ising_pt* pt, int sweeps_per_swap, int rounds);
/* n_sweeps sweeps of every replica at its current temperature without exchange: the
 * "relax each domain" loop of src/PT.f90:276-287. */
int ising_pt_relax(ising_pt* pt, int n_sweeps);
/* Test hook of the persistent octant engine (octant meshes, sweep_kernel 3): during the next
 * ising_pt_run call every dependency wait of the first class change gives up after wait_ms
 * milliseconds (a count nothing reaches); the call returns ISING_ERR_TIMEOUT, the context
 * stays usable, and ising_pt_resync restores the running energies.  No reference
 * counterpart. */
int ising_pt_inject_stall(ising_pt* pt, int wait_ms);
/* Launch schedule of a round: replicas per L2 group, colour-pass launches per round of
 * sweeps_per_swap sweeps, and which colour-pass kernel runs (1 register, 2 TMA-staged,
 * 0 the stencil kernel of the greedy or octant colouring, 3 the octant kernel with the
 * stencil resolved per class, 4 the persistent octant engine, 5 the sublattice classes of
 * BCC meshes, 6 the octant kernel with a pair of sites per thread).  No reference
 * counterpart. */
int ising_pt_schedule(const ising_pt* pt, int sweeps_per_swap, int* l2_group, int* pass_launches,
                      int* kernel);
/* temperature slot -> replica (TemperatureMeshArray(i, :), src/PT.f90:58) */
int ising_pt_permutation(const ising_pt* pt, int* temp_to_replica);
/* running FP64 energies and magnetisation vectors by replica */
int ising_pt_energies(const ising_pt* pt, double* e_per_replica, double* m_per_replica);
/* recompute the running accumulators from the spins (periodic FP64 resync) */
int ising_pt_resync(ising_pt* pt);
/* attempts and accepts per neighbour pair (t, t+1), n_temps-1 entries each */
int ising_pt_swap_stats(const ising_pt* pt, uint64_t* attempts, uint64_t* accepts);
/* Recorded series by temperature slot (the replica holding slot t at each recorded
 * sweep): E, |M| = |sum S|/N, Q_mid (slice nz/2) and Q_mean (mean over slices).
 * out is n_temps x record_capacity x 4; *n_recorded gives the filled length. */
int ising_pt_series(const ising_pt* pt, double* out, int* n_recorded);

/* ---------------------------------------------------------------- batched ensembles
 * Many independent PT ensembles (one per parameter slot of src/PT.f90:147-176, which the
 * reference runs one after another per MPI rank) of uneven lattice sizes and Hamiltonians,
 * all replicas advanced by ONE persistent kernel per launch: sweeps, running-sum folds and
 * exchanges of every ensemble, replayed from a CUDA graph.  Each ensemble is a
 * colour-separated simple-cubic mesh (even nx, ny; nz % 4 == 0; shell 1 only).  The per-site
 * updates, Philox keys and exchange decisions are those of ising_pt_* on the same mesh,
 * seed and ensemble id.  The engine issues all work on its own stream (or the one
 * ising_ensembles_set_stream gives); the meshes must not be used elsewhere meanwhile and
 * must outlive the engine (destroy the engine first). */
typedef struct ising_ensembles ising_ensembles;

typedef struct {
    ising_mesh* mesh;
    int n_temps;              /* replicas 0..n_temps-1 of mesh take part */
    const double* betas;      /* n_temps inverse temperatures by slot */
    ising_params params;
    uint32_t ensemble;        /* Philox key component (< 2^24), distinct per ensemble */
} ising_ensemble_desc;

#define ISING_ENS_ORDER_PHASE 0   /* queue by colour pass: every ensemble's pass p, then p+1 */
#define ISING_ENS_ORDER_GROUPS 1  /* replica groups of ~group_bytes run a whole round in turn
                                     (the group's spins stay resident in L2) */
#define ISING_ENS_ORDER_WAVE 2    /* colour passes as a wavefront: pass p visits chunk
                                     (p + i) mod nch at step 3p + i, so consecutive passes
                                     follow each other through the lattice */

typedef struct {
    uint64_t seed;
    int move;                 /* ISING_MOVE_UNIFORM or ISING_MOVE_BALL, all ensembles */
    double r;
    int scheme;               /* ISING_PT_EVEN_ODD or ISING_PT_RANDOM_PAIRS */
    int resync_every;         /* rounds between FP64 energy resyncs (0 = never) */
    int wait_timeout_ms;      /* bound of every in-kernel wait (0 = 2000) */
} ising_ensembles_options;

#define ISING_ENS_LOADER_REGISTERS 0   /* each thread loads its sites' neighbours from global memory */
#define ISING_ENS_LOADER_STAGED 1      /* rows staged in shared memory by TMA copies (every ensemble
                                          with nz = 128 and nx % 4 == 0; whole groups of 4 x-planes
                                          per task; 256-thread blocks) */
#define ISING_ENS_LOADER_FUSED 2       /* both colour passes of a sweep in one pass over memory:
                                          a task updates one sweep of a chunk of x-planes (one
                                          thread row per plane plus a halo plane on either side;
                                          block_threads 128..512 and >= nz) and a y-segment
                                          (chunk_pairs / chunk width / (nz/4) rows), reading one
                                          spin buffer and writing a second one the engine
                                          allocates; sweeps_per_swap must be even.  Bit-identical
                                          to the other loaders. */

/* One schedule: block size, target site pairs per task, queue order, group size, loader. */
typedef struct {
    int block_threads;        /* 64..256 (fused loader 128..512), whole warps */
    int chunk_pairs;          /* site pairs of one colour per task (whole x-planes) */
    int order;                /* ISING_ENS_ORDER_* */
    int64_t group_bytes;      /* ISING_ENS_ORDER_GROUPS: spin bytes per replica group */
    double ms_per_round;      /* autotuner output: measured time per round */
    int loader;               /* ISING_ENS_LOADER_* */
} ising_ensembles_schedule_t;

/* No reference counterpart (the reference has no batched form). */
int ising_ensembles_create(int n_ensembles, const ising_ensemble_desc* desc,
                           const ising_ensembles_options* opt, ising_ensembles** out);
int ising_ensembles_destroy(ising_ensembles* s);
int ising_ensembles_set_stream(ising_ensembles* s, void* cuda_stream);
/* rounds x [sweeps_per_swap sweeps of every replica of every ensemble, then each
 * ensemble's exchange]: the iteration loop of src/PT.f90:219-273 for all slots at once. */
int ising_ensembles_run(ising_ensembles* s, int sweeps_per_swap, int rounds);
int ising_ensembles_set_schedule(ising_ensembles* s, const ising_ensembles_schedule_t* sched);
/* current schedule, persistent grid size and tasks per colour pass (all replicas) */
int ising_ensembles_get_schedule(const ising_ensembles* s, ising_ensembles_schedule_t* sched,
                                 int* grid_blocks, int64_t* tasks_per_pass);
/* Times candidate schedules (each trial runs warm-up and rounds_per_trial ordinary rounds
 * of the chain) and keeps the fastest; trials may be NULL. */
int ising_ensembles_autotune(ising_ensembles* s, int sweeps_per_swap, int rounds_per_trial,
                             ising_ensembles_schedule_t* trials, int max_trials, int* n_trials);
int ising_ensembles_permutation(const ising_ensembles* s, int ensemble_index, int* temp_to_replica);
int ising_ensembles_energies(const ising_ensembles* s, int ensemble_index, double* e_per_replica,
                             double* m_per_replica);
int ising_ensembles_swap_stats(const ising_ensembles* s, int ensemble_index, uint64_t* attempts,
                               uint64_t* accepts);
int ising_ensembles_resync(ising_ensembles* s);
/* Recompute every replica's FP64 energy and magnetisation accumulators from its spins after
 * each `every` rounds of ising_ensembles_run, counted from this call (0: never); the option
 * resync_every of ising_ensembles_create, re-armed.  No reference counterpart: the reference
 * recomputes TotalHeisenbergEnergy at every exchange (src/PT.f90:251-254). */
int ising_ensembles_set_resync(ising_ensembles* s, int every);
/* Test hook for the bounded waits: in the next run, rounds >= 1 of ensemble_index wait for
 * a flag that nothing sets, so that run returns ISING_ERR_TIMEOUT after wait_timeout_ms;
 * the engine then resynchronises its accumulators and stays usable. */
int ising_ensembles_inject_stall(ising_ensembles* s, int ensemble_index);

/* ---------------------------------------------------------------- CSV outputs */
/* write_spins_to_file(chainMesh, filename, append, include_header, frame_index)
 * (src/LLG.f90:93-172): "x,y,z,Sx,Sy,Sz" with ES22.14; frame_index < 0 means absent. */
int ising_write_spins_csv(const ising_mesh* mesh, int replica, const char* path, int append,
                          int include_header, int frame_index);
/* The data_<J>_<D>_<B>_<T>.csv record of src/PT.f90:318-362 (header, F0.4/F0.10 and
 * F0.4/I0.4/F0.2 formats) and its file name (PT.f90:337-341). */
int ising_write_pt_data_csv(const char* path, double J, double D, double B, double T,
                            double wnd_mid, int sk_mid, double wnd_spread, const double m[3]);
int ising_pt_file_tag(char* buf, size_t cap, double J, double D, double B, double T);
/* write_winding_number_density_interpolated (rsp:502-540): the density file of the fine grid
 * of every slice (positions from the fine indices, as in the reference). */
int ising_write_winding_density_interpolated_csv(const ising_mesh* mesh, int replica, const char* path);
/* frame file name of the annealing driver: trim(output_dir)//"/frame_"//I5.5//".csv"
 * (src/ISING.f90:218). */
int ising_frame_filename(char* buf, size_t cap, const char* output_dir, int index);
/* info.txt of the annealing driver (src/ISING.f90:232-237): frame count, then numCellsX and
 * the lattice parameter, blank-separated as the visualisation scripts parse it. */
int ising_write_frame_info(const char* path, int num_frames, int num_cells_x, float lattice_param);
/* write_winding_number_density (rsp:544-580): "x,y,z,Winding_Density" with F0.8; the
 * densities come from one device pass, the records are formatted on all host threads. */
int ising_write_winding_density_csv(const ising_mesh* mesh, int replica, const char* path);

/* ---------------------------------------------------------------- learned patch proposal */
/* 3^3 convolution of a channel-last BF16 grid (nwin windows of Gi^3 cells x C channels, C = 8
 * or 32) onto Go^3 output cells with zero padding pad, as an implicit GEMM on the tensor cores:
 * out(row, n) = bias[n] + sum_{o, ch} in[window][cell(row) + offset(o) - pad][ch] w[n][o C + ch]
 * with K = 27 C rounded up to 16, rows = nwin Go^3 (FP32 rows in c and/or GELU'd BF16 rows in
 * o_bf16).  loader: 0 = automatic, 1 = register-staged operands, 2 = TMA copies (C = 32,
 * Go = 4 only).  No reference counterpart (the learned proposal's network). */
int ising_conv3_bf16(const void* in, int C, int Gi, int Go, int pad, int nwin, const void* w, int ldb, int N,
                     const float* bias, float* c, int ldc, void* o_bf16, int ldo, int gelu, int loader,
                     void* stream);
/* Tensor-core GEMM on device buffers (no reference counterpart): c / o_bf16 (M x N) =
 * a (M x K, BF16, K contiguous) * b (N x K, BF16)^T (+ bias[N]); o_bf16 gets GELU(tanh form)
 * of the sum when gelu = 1.  N multiple of 16 up to 256, K multiple of 16, row pitches
 * multiples of 8; a must hold ceil(M/128)*128 readable rows.  stream is a cudaStream_t
 * (NULL = legacy default stream); the call synchronises it. */
int ising_bf16_gemm(const void* a, int lda, const void* b, int ldb, int M, int N, int K, const float* bias,
                    float* c, int ldc, void* o_bf16, int ldo, int gelu, void* stream);

/* The proposal network (no reference counterpart; the reference proposes single-spin moves
 * only, src/energyMin.f90:49-68).  Input windows are FP32 device arrays [n][3][8][8][8]
 * (component, then window site (i, j, k) = lattice site (px-2+i, py-2+j, pz-2+k) of a patch
 * with lowest corner (px, py, pz)); output [n][64][4] = (mu_x, mu_y, mu_z, log sigma) per
 * patch site (i, j, k of the 4^3 patch, k fastest).  Parameters are FP32 in PyTorch conv3d
 * order: W1[32][3][3][3][3], b1[32], W2[32][32][3][3][3], b2, W3, b3, Wh[4][32], bh[4]. */
typedef struct ising_net ising_net;
int ising_net_create(int device, int max_batch, uint64_t seed, ising_net** out);
int ising_net_destroy(ising_net* net);
int ising_net_param_count(void);
int ising_net_set_params(ising_net* net, const float* host_params);
int ising_net_get_params(const ising_net* net, float* host_params);
int ising_net_forward(ising_net* net, const float* d_windows, int n, float* d_out);
/* mean Gaussian NLL of target patch spins d_targets [n][64][3] (tangent rotation from the
 * window's patch spins) and its gradient (host_grads may be NULL) */
int ising_net_loss_grad(ising_net* net, const float* d_windows, const float* d_targets, int n, double* loss,
                        float* host_grads);
/* one Adam step on that loss */
int ising_net_train_step(ising_net* net, const float* d_windows, const float* d_targets, int n, double lr,
                         double* loss);

/* The learned patch move on a PT object (simple-cubic mesh, nx, ny, nz divisible by 8; no
 * reference counterpart): one class `colour` (0..7) of the 2x2x2 colouring of 4^3 blocks,
 * shifted by (offx, offy, offz), on the replicas holding temperature slots 0..slots-1
 * (slots = 0: all).  Each patch gets a network proposal and an exact Metropolis-Hastings
 * accept; the running FP64 energies and magnetisations follow the accepted patches. */
int ising_pt_patch_step(ising_pt* pt, ising_net* net, int colour, int offx, int offy, int offz, int slots);
/* Per-slot step scale a and drift weight l of the patch move: the tangent move becomes
 * a * (l P_s(mu) + sigma eps), still an exact MH proposal.  scale_per_slot holds n_temps
 * positive values, or NULL for a = 1; l = 1 uses the mean rotation as predicted. */
int ising_pt_patch_set_scale(ising_pt* pt, const float* scale_per_slot, float drift);
/* windows per patch step (slots x (nx/8)(ny/8)(nz/8)) */
int ising_pt_patch_count(const ising_pt* pt, int slots, int64_t* n_windows);
/* Training samples from the current PT state: the windows of one colour class (device
 * [n][3][8][8][8]) and, as targets (device [n][64][3]), their patches after n_local
 * Metropolis sweeps of the patch with the halo fixed at the replica's temperature. */
int ising_pt_patch_samples(ising_pt* pt, int colour, int offx, int offy, int offz, int slots, int n_local,
                           float* d_windows, float* d_targets);
/* Inspection of the last patch step's first n windows (its first batch): windows x and x'
 * ([n][3][8][8][8]), log q(x'|x) per window, and, for the first n windows of the step, the
 * energy change and the accept flag.  Any pointer may be NULL. */
int ising_pt_patch_last(const ising_pt* pt, int n, float* win, float* winp, double* lqf, double* dE, int* accepted);
/* per temperature slot: sum over accepted patch moves of sum_i |s_i' - s_i|^2 since creation
 * (the expected squared jump distance is this over the proposals) */
int ising_pt_patch_jump(const ising_pt* pt, double* sq_jump_per_slot);
/* patch moves proposed and accepted per temperature slot since creation */
int ising_pt_patch_stats(const ising_pt* pt, uint64_t* proposed, uint64_t* accepted);

#ifdef __cplusplus
}
#endif
#endif /* ISING_GPU_H */
