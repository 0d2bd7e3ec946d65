// ensembles.h -- device-side description of the persistent multi-ensemble PT engine.
//
// Work is a queue of tasks, one per (ensemble e, replica r, phase, chunk): a phase is one
// colour pass (phase p of a round is colour p & 1 of sweep p >> 1), a chunk is P consecutive
// x-planes of the colour-separated layout.  A task may start when its own chunk and the two
// x-neighbour chunks (cyclic) have finished the previous phase, and, for the first phase of
// a round, when ensemble e has finished the previous round's exchange.  The queue order
// (host-built table) puts every task after all tasks it waits for, so a block only ever waits
// for tasks that running blocks hold and the kernel needs no co-residency guarantee.  The
// last task of a round of ensemble e folds the partial sums and runs the exchange in-kernel.
#pragma once
#include <cuda.h>   // CUtensorMap

#include "sweep_cb.cuh"

namespace isg {

constexpr int kMaxEnsembles = 16;   // compile-time slots of the kernel's ensemble switch
constexpr int kEnsMaxThreads = 256;

struct EnsDev {
    CbGeom g;                    // geometry and Hamiltonian for the pair update
    float* spins;                // replica 0 of the mesh
    uint32_t N;                  // atoms per replica
    FastDiv divNY;
    FastDiv divTX;               // W / 2 lanes per packed row
    uint32_t P;                  // x-planes per chunk
    uint32_t nch;                // chunks per replica
    uint32_t rb;                 // thread rows per block: threads / (W / 2)
    uint32_t nseg, seg_len;      // y-segments per plane in a task, rows per segment
    FastDiv divSeg;              // by nseg
    uint32_t st_nseg, st_seg_len;   // staged loader: y-segments per group of kStG planes, rows per segment
    float* spins_b;              // fused loader: the second spin buffer (same layout as spins)
    uint32_t fnch, fnseg;        // fused loader: chunks of x-planes, y-segments (nch = fnch * fnseg units)
    uint32_t fnp;                // fused loader: thread rows per block (widest chunk + 2 halo planes)
    int n_rep;                   // replicas 0..n_rep-1 (= temperature slots)
    double* beta_rep;
    uint32_t* sweep_ctr;         // the mesh's per-replica sweep counters
    double* partials;            // [n_rep][nch][4]: dE, dMx, dMy, dMz of the running round
    uint32_t* done;              // [n_rep][nch]: phases finished in this launch
    uint32_t* ready;             // rounds of this launch whose exchange is finished
    unsigned long long* fin;     // final-phase tasks finished in this launch
    Acc4* acc;
    const double* beta_t;
    int* t2r;
    int* r2t;
    unsigned long long* stats;
    uint32_t* round_ctr;
};

// Staged loader (schedule loader 1; W = 64 only): a sub-block of kStG warps marches kStG
// consecutive x-planes (one warp per plane) along y in lockstep.  For each row y a ring stage
// receives, by two tiled TMA copies, the own colour's rows (planes x0 .. x0+kStG-1, all three
// components) and the other colour's row y+1 of planes x0-1 .. x0+kStG; rows y-1 and y of
// the other colour are the previous two stages.  A separate copy warp issues the copies.
constexpr int kStG = 4;
constexpr int kStSub = 2;                  // sub-blocks of compute warps per block
constexpr int kStThreads = kStSub * kStG * 32 + 32;   // the compute warps and one copy warp
constexpr int kStStages = 7;               // ring stages per sub-block
constexpr uint32_t kStNxtFloats = 3u * (kStG + 2) * 64u;   // [3][kStG+2][64]
constexpr uint32_t kStOwnFloats = 3u * kStG * 64u;         // [3][kStG][64]
constexpr uint32_t kStStageFloats = kStNxtFloats + kStOwnFloats;
constexpr uint32_t kStSmemBytes = kStSub * kStStages * kStStageFloats * 4u + 2u * kStSub * kStStages * 8u + 128u;

// Fused loader (schedule loader 2): one pass per sweep over ping-pong buffers, a block of up to
// kFuMaxThreads threads holding one thread row per x-plane of a chunk plus two halo planes.
constexpr int kFuMaxThreads = 512;

// Tensor maps of one ensemble's spins, dims (entry, y, x, colour, 3 replica + component):
// next = box {64, 1, kStG+2, 1, 3}, own = {64, 1, kStG, 1, 3}, ctr = {64, 1, kStG, 1, 1},
// halo = {64, 1, 1, 1, 1} (ctr and halo serve plane groups whose x-halo wraps around).
struct alignas(64) EnsMaps {
    CUtensorMap next, own, ctr, halo;
};

struct EnsParams {
    EnsMaps maps[kMaxEnsembles];   // staged loader only
    EnsDev e[kMaxEnsembles];
    int n_ens;
    const uint2* table;          // one round: x = e << 24 | r, y = phase << 16 | chunk
    uint32_t tasks_per_round;
    uint32_t rounds;
    uint32_t k;                  // sweeps per round
    uint32_t* head;              // queue position
    uint32_t* abort;             // set when a wait gives up; every block then stops
    uint32_t* where;             // 1 + task id of the first wait that gave up
    int* status;
    uint64_t wait_ns;            // bound of every wait
    int scheme;
    int stall_ens;               // test hook: round >= 1 of this ensemble waits for a flag nothing sets
    uint64_t seed;
    uint32_t rk[20];             // Philox round keys of seed
};
static_assert(sizeof(EnsParams) < 32000, "kernel parameter block too large");

// loader: 0 registers, 1 staged, 2 fused (smem = dynamic shared memory of the fused kernel)
int launch_ensembles(const EnsParams& P, int move, int dmi, bool has_k, int loader, int threads, int grid,
                     size_t smem, cudaStream_t s);
// kernel instantiations, one translation unit per move kind (dmi in 1..3: 1 bulk,
// 2 interfacial about z, 3 tabulated per bond direction)
const void* ensembles_kernel_uniform(int dmi, bool has_k, int loader);
const void* ensembles_kernel_ball(int dmi, bool has_k, int loader);
int ensembles_blocks_per_sm(int move, int dmi, bool has_k, int loader, int threads, size_t smem, int* out);
// the staged loader's tensor maps for one ensemble (spins of n_rep replicas of an
// nx x ny x 128 colour-separated mesh); false if the driver refuses one
bool ensembles_encode_maps(float* spins, int nx, int ny, int n_rep, EnsMaps* m);

}  // namespace isg
