// internal.h -- host-side structures of libisinggpu (not part of the C-ABI).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/ising_gpu.h"
#include "device.cuh"

namespace isg {

// ---------------------------------------------------------------- errors
void set_error(const std::string& msg);
int fail(int status, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);
// the driver's cuTensorMapEncodeTiled (nullptr if the driver has none), looked up once
void* tensor_map_encoder();
#define ISG_CUDA(call)                                              \
    do {                                                            \
        cudaError_t e_ = (call);                                    \
        if (e_ != cudaSuccess) return ::isg::cuda_fail(e_, #call);  \
    } while (0)

// ---------------------------------------------------------------- lattice compiler
// A neighbour of sublattice i expressed as a cell offset plus target sublattice, with the
// minimum-image bond vector r_j - r_i.  Because the periodic mesh is translation
// invariant, one list per sublattice (built at cell 0) describes every atom.
struct NbrSlot {
    int dx, dy, dz, sub;
    double r[3];
};

struct Lattice {
    int nx = 0, ny = 0, nz = 0, nsub = 0, nshells = 2;
    int64_t ncells = 0, natoms = 0;
    double a = 0, b = 0, c = 0;
    double av[3], bv[3], cv[3], ar[3], br[3], cr[3];
    std::vector<float> frac;                      // nsub x 3
    std::vector<std::vector<NbrSlot>> shell[2];   // per sublattice, shells 1 and 2
    std::vector<std::vector<NbrSlot>> legacy;     // per sublattice, legacy NeighborList
    std::vector<NbrSlot> deriv;                   // [sub*6 + d*2 + side]
    bool deriv_ok = true;

    // position of atom (cell, sub) as real(4), as makeChainMesh stores it
    void position(int64_t atom, float out[3]) const;
    int64_t atom_of(int ix, int iy, int iz, int sub) const {
        return (((int64_t)ix * ny + iy) * nz + iz) * nsub + sub;
    }
    void cell_of(int64_t atom, int* ix, int* iy, int* iz, int* sub) const;
    int64_t neighbour_atom(int64_t atom, const NbrSlot& s) const;
};

// Builds a Lattice; returns ISING_OK or an error status (message set).
int build_lattice(const float* frac, int nsub, int nx, int ny, int nz, double a, double b,
                  double c, double ab_deg, double bc_deg, double ca_deg, double shell_tol,
                  int n_shells, Lattice* out);

// Greedy colouring of the bond graph of the active shells (shell 1 always, shell 2 when
// use_shell2).  Returns colour per atom and the number of colours; verifies that every
// class is an independent set.
int greedy_colouring(const Lattice& L, bool use_shell2, std::vector<int>* colour, int* ncol);

// True if the mesh is simple cubic with the six axis neighbours as shell 1 and even
// extents, so the 2-colour checkerboard fast path applies.
bool is_checkerboard_sc(const Lattice& L);

// Sublattice groups of the octant colouring (class = cell octant x sublattice group) of a
// general crystal; false when the octant colouring does not apply (odd extents, or a bond of
// shells 1-2 between two sites of one sublattice at an all-even non-zero cell offset).
// class_of_group: each group's shell-1 class (groups of a class are consecutive; a class is
// free of shell-1 bonds in all 8 octants), or empty when shell 1 does not allow them.
bool octant_groups(const Lattice& L, std::vector<int>* group, int* ngroups,
                   std::vector<int>* class_of_group = nullptr);
// classes of the octant blocks (octant o, sublattice s) for the active shells, each as the
// ascending list of o * nsub + s (a DSatur colouring of the block graph)
bool octant_block_classes(const Lattice& L, bool shell2, std::vector<std::vector<int>>* out);
// two sublattices joined only to each other by the first shell, 8 neighbours in cells
// base + {0,1}^3 (layout 3); base[s] per sublattice
bool bipartite_pair(const Lattice& L, int base[2][3]);

// ---------------------------------------------------------------- device-side handle
struct Colouring {
    int ncol = 0;
    std::vector<int> host_colour;
    std::vector<int> class_start;   // ncol + 1
    int* d_sites = nullptr;         // atoms grouped by class
    // octant layout: the blocks (octant, storage rank) of each class as octant << 4 | rank,
    // ascending (storage order)
    std::vector<std::vector<uint8_t>> oct_blocks;
};

struct DeviceStencil {
    Slot* d_slots = nullptr;        // kMaxSub * kMaxSlots
    int* d_count = nullptr;         // kMaxSub
    bool built = false;
};

}  // namespace isg

struct ising_mesh {
    isg::Lattice lat;
    int device = 0;
    int n_replicas = 0;
    cudaStream_t stream = nullptr;       // stream all work is issued on
    cudaStream_t own_stream = nullptr;   // the handle's own stream
    float* d_spins = nullptr;            // [R][3][natoms] FP32 SoA planes
    uint32_t* d_sweep = nullptr;         // per-replica sweep counters
    std::vector<uint32_t> h_sweep;       // host mirror of d_sweep
    double* d_scratch = nullptr;         // small per-call device buffer (kScratchDoubles)
    double* h_pinned = nullptr;          // pinned host mirror of d_scratch
    int* d_status = nullptr;             // device status word
    double* d_beta = nullptr;            // per-replica beta for single-replica sweeps
    double* d_staging = nullptr;         // 3N doubles for host-layout spin transfers
    size_t staging_size = 0;
    double* d_winding_tmp = nullptr;     // per-slice winding results
    bool checkerboard = false;
    isg::Layout layout{};                // storage order of the spin planes
    std::vector<int> oct_rank0;          // octant layout: first storage rank of each sublattice group (+ end)
    isg::Colouring colour[2];            // [0]: shell 1 bonds, [1]: shells 1+2
    // cached device stencils keyed by the Hamiltonian that filled their weights
    isg::Slot* d_slots = nullptr;
    int* d_slot_count = nullptr;
    int* d_plaq = nullptr;               // winding plaquette offsets (4 x {dx,dy,sub})
    int sclx = 10, scly = 10;            // fine-grid scale factors (makeChainMesh defaults)
    void* sky = nullptr;                 // skyrmion-counting workspace, made on first use
    void* xfer = nullptr;                // asynchronous spin transfers (streams, per-replica staging)
    void* demag = nullptr;               // demagnetising-field workspace, made on first use
    uint32_t* d_oct_sync = nullptr;      // octant engine: [n_replicas][nx/2] counters + head + abort
    int bip_base[2][3] = {{0, 0, 0}, {0, 0, 0}};   // layout 3: first-shell cell offsets per sublattice
    std::vector<int> oct_class0;         // octant layout: first storage rank of each shell-1 class
                                         // (+ end), empty when there are none; without J' a sweep
                                         // is one class (all 8 octants) after another
};

namespace isg {
// Frees the skyrmion-counting workspace of a mesh (called by ising_mesh_destroy).
void skyrmion_release(ising_mesh* m);
// Demagnetising field (calculate_demagnetisation_field, src/reciprocalSpaceProcesses.f90:202-281)
// of one replica, enqueued on the mesh's stream: FP64 per atom in reference order
// (demag_field64, [3][natoms]) and/or FP32 in the storage order of the spins (demag_field32).
int demag_enqueue(ising_mesh* m, int replica, bool want64, bool want32);
const double* demag_field64(const ising_mesh* m);
const float* demag_field32(const ising_mesh* m);
// sum over atoms of S . H (FP64) for the field last computed into demag_field64 (synchronous)
int demag_dot(ising_mesh* m, int replica, double* out);
void demag_release(ising_mesh* m);
constexpr double kMu0 = 1.25663706127e-6;   // mu_0 of src/constants.f90:15
// Waits for the mesh's asynchronous spin transfers (ising_spins_*_async) still in flight and
// reports invalid uploaded spins; a no-op when none are.  Every entry point that reads or
// writes a mesh's spins calls it first.
int mesh_settle(const ising_mesh* m);
}  // namespace isg

namespace isg {
constexpr int kScratchDoubles = 1 << 16;
constexpr double kL2GroupBytes = 64.0e6;   // replica group size of the paired colour schedule

// Kernel launchers.
// Colour-separated checkerboard sweep (sweep_cb.cu): up to two segments per launch, each a
// replica range, a colour and a sweep offset.
struct CbSeg {
    int rep_first, n_rep, colour;
    uint32_t sweep_offset;
};
struct CbLaunch {
    float* spins;          // replica 0 of the mesh
    int64_t natoms;
    int nx, ny, nz;
    CbSeg seg[2];
    int n_seg;
    const double* beta_rep;
    const uint32_t* sweep_ctr;
    uint64_t seed;
    uint32_t ensemble;
    float r;
    HamDev ham;
    double* partials;
    int slots_per_rep;
    int* status;
};
int cb_slots_per_rep();
int launch_cb_sweep(const CbLaunch& a, int move, int dmi_kind, cudaStream_t s);
// TMA-staged variant (sweep_tma.cu): nz % 8 == 0
bool cb_tma_supported(int nx, int ny, int nz);
int cb_tma_slots_per_rep(int nx, int ny, int nz);
int launch_cb_tma(const CbLaunch& a, int move, int dmi_kind, cudaStream_t s);

struct GeneralLaunch {
    float* spins;
    int64_t natoms;
    int nx, ny, nz, nsub;
    int n_rep, rep_first;
    const double* beta_rep;
    const uint32_t* sweep_ctr;
    uint32_t sweep_offset;
    uint64_t seed;
    uint32_t rk[20];         // Philox round keys of seed (philox_round_keys)
    uint32_t ensemble;
    int move;
    float r;
    HamDev ham;
    StencilDev st;
    Layout layout;
    const int* sites;      // atoms of this colour class
    int n_sites;
    double* partials;
    int slots_per_rep;
    int slot_base;         // class offset into the slot range
    int* status;
    const float* demag;    // demagnetising field of the (single) replica in storage order, or null
    float mu0;             // its factor in the local field: h -= mu0 H
    int oct_maxcnt;        // octant layout: largest stencil of a sublattice when every neighbour's
                           // packed offset needs at most one periodic wrap (k_octant_fast), else 0
};
int launch_general_colour(const GeneralLaunch& a, cudaStream_t s);
// One class (octant, sublattice group) of an octant-layout mesh: sites of storage ranks
// [rank0, rank0 + nrank) of that octant (a.sites and a.n_sites unused).
// One colour class of an octant-layout mesh as a list of blocks (cell octant o, storage rank
// r), each code o << 4 | r; the blocks' sites share no bond.
constexpr int kMaxOctBlocks = 8 * kMaxSub;
struct OctBlocks {
    int n;
    uint8_t code[kMaxOctBlocks];
};
// the class in one launch, or in runs of blocks whose stencils fit 48 KB of shared memory;
// partial slots from a.slot_base, octant_class_slots of them
int launch_octant_class(const GeneralLaunch& a, const OctBlocks& b, cudaStream_t s);
int octant_class_slots(int64_t q8, int nblocks, int maxcnt);
int octant_class_launches(int nblocks, int maxcnt);
int octant_slots_for(int64_t n_sites, bool fast);   // partial-sum slots (blocks) of one class launch
// The octant sweeps of a PT round as ONE persistent launch: tasks (sweep, class, replica,
// packed x-plane) in phase-major queue order, each waiting (bounded) until the planes within
// `reach` of its own have finished the previous phase.  Partial sums: one slot per (replica,
// plane), so slots_per_rep >= hx.
struct OctEngineLaunch {
    uint32_t* done;          // [n_rep][hx] phases completed in this launch (zeroed before it)
    uint32_t* head;          // task queue head (zeroed before it)
    uint32_t* abort;         // raised by a wait that gives up (zeroed before it)
    int n_sweeps, reach;     // sweeps, dependency reach in packed x-planes
    int ncls, maxnb;         // classes per sweep, most blocks in a class
    uint8_t code[kMaxOctBlocks];        // the blocks of every class, class after class
    uint8_t start[kMaxOctBlocks + 1];   // class c: code[start[c] .. start[c + 1])
    uint64_t wait_ns;        // bound of every wait
    int grid;                // persistent blocks
    int stall;               // test hook: the tasks of phase 1 wait for a count nothing reaches
};
int launch_octant_engine(const GeneralLaunch& a, const OctEngineLaunch& e, cudaStream_t s);
// One sublattice class of a layout-3 mesh (BCC without J'): the first shell of sublattice
// `sub` as 8 bonds to the other sublattice's cells base + (a, b, c), a, b, c in {0, 1}.
struct BipClass {
    int base[3];
    float w[8];              // bond (a, b, c) at index a * 4 + b * 2 + c
    float D[8][3];
};
int launch_bip_sweep(const GeneralLaunch& a, const BipClass& c, int sub, cudaStream_t s);
int bip_slots_per_class();   // partial-sum slots (blocks) of one class launch
int octant_engine_grid(int* blocks);
int general_slots_for(int n_sites);

struct ReduceLaunch {
    const float* spins;
    int64_t natoms;
    int nx, ny, nz, nsub;
    int n_rep;
    HamDev ham;            // Bz already multiplied by the zeeman factor
    StencilDev st;         // slots used for the energy (weights 0.5 applied in kernel)
    Layout layout;
    double* out;           // [rep][4]: E, Mx, My, Mz
    double* block_tmp;     // [rep][blocks][4]
    int blocks_per_rep;
};
int launch_energy_mag(const ReduceLaunch& a, cudaStream_t s);
int energy_blocks_for(int64_t natoms);

int launch_fold_partials(double* partials, int slots_per_rep, int n_rep, Acc4* acc,
                         cudaStream_t s);

struct WindingLaunch {
    const float* spins;
    int64_t natoms;
    int nx, ny, nz, nsub;
    int n_rep;
    const int* plaq;       // 4 entries of (dx, dy, dz, sub) relative to sublattice nsub-1
    Layout layout;
    double* out;           // [rep][nz]
    int fp64;
    double* dens;          // optional plaquette densities [rep][slice][ny][nx] (nx fastest), or NULL
    int z0, nzc;           // slices z0 .. z0+nzc-1 (nzc == 0: all nz slices)
};
int launch_winding(const WindingLaunch& a, cudaStream_t s);

struct LocalLaunch {
    const float* spins;    // one replica
    int64_t natoms;
    int nx, ny, nz, nsub;
    HamDev ham;
    StencilDev st;
    Layout layout;
    const int64_t* atoms;
    const double* sprop;   // n x 3
    double* old_e;
    double* new_e;
    int n;
    const double* demag_H; // demagnetising field per atom, reference order [3][natoms], or null
};
int launch_local_energy(const LocalLaunch& a, cudaStream_t s);

int launch_init_uniform(float* spins, int64_t natoms, const Layout& L, int n_rep, uint64_t seed,
                        uint32_t ensemble, cudaStream_t s);
int launch_advance(uint32_t* ctr, int n, uint32_t by, cudaStream_t s);
int launch_spins_from_f64(const double* in, float* out, int64_t natoms, const Layout& L, int* status,
                          cudaStream_t s);
int launch_spins_to_f64(const float* in, double* out, int64_t natoms, const Layout& L, cudaStream_t s);

struct ExchangeLaunch {
    int n;                       // temperature slots
    const double* beta_t;        // per slot
    double* beta_rep;            // per replica (updated)
    int* t2r;
    int* r2t;
    const Acc4* acc;             // per replica
    unsigned long long* stats;   // [2][n-1]: attempts, accepts
    uint32_t* round;             // device round counter (advanced)
    uint64_t seed;
    uint32_t ensemble;
    int scheme;
};
int launch_exchange(const ExchangeLaunch& a, cudaStream_t s);

struct RecordLaunch {
    const Acc4* acc;
    const double* q;     // [rep][nz] winding per slice
    const int* t2r;      // temperature slot -> replica
    int nz;
    int n_rep;
    int64_t natoms;
    double* series;      // [slot][cap][4]
    int cap;
    int* count;          // device count (advanced)
};
int launch_record(const RecordLaunch& a, cudaStream_t s);

// host helpers shared with the allocation-free entry point (capi.cu)
int fill_query_stencil_host(const ising_mesh* m, const ising_params& p, bool legacy, Slot* slots, int* cnt);
HamDev ham_of(const ising_params& p);
int check_params(const ising_params* p);

}  // namespace isg
