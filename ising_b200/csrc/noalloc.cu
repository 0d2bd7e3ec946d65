// noalloc.cu -- total energy of one replica without allocating device memory.
//
// ising_total_energy obtains the scratch for its per-block partial sums with cudaMalloc on
// every call.  Some callers cannot do that: a driver loop that must not stall concurrent
// streams (cudaFree synchronises the whole device), code issued while another thread
// captures a CUDA graph in global mode (cudaMalloc is not permitted then), or an embedding
// application that reserves all device memory up front.  This variant keeps the scratch in a
// file-scope __device__ array instead: every device that loads the library holds
// kNoAllocScratchDoubles doubles (128 KiB + 32 B) until the process exits, and the largest
// replica it accepts has 4096 x 4096 = 16,777,216 atoms (4096 reduction blocks of 4096 sites).
//
// The array is shared by every call on a device and keeps the contents of the last call.
// Nothing in it needs clearing: each call overwrites every partial it later reads.  Two
// calls whose work overlaps on the GPU (different streams, or different host threads) race
// on the array; issue them one after another.
//
// The first call on a device resolves the array's device address with cudaGetSymbolAddress
// (with that device current); make that first call before any stream capture begins.  The
// address is kept for the life of the process: a cudaDeviceReset unloads the module and makes
// it stale, so this entry point must not be used on a device after that device was reset.
#include <mutex>

#include "internal.h"

namespace isg {
namespace {

constexpr int kNoAllocMaxBlocks = 4096;                 // block partials of one replica
constexpr int kNoAllocScratchDoubles = kNoAllocMaxBlocks * 4 + 4;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

double* g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mu;

// device address of g_noalloc_scratch on the current device `dev`, resolved once
int scratch_for(int dev, double** out) {
    if (dev < 0 || dev >= kMaxDevices) return fail(ISING_ERR_ARG, "device index beyond the supported range");
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_scratch_addr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_addr[dev];
    return ISING_OK;
}

}  // namespace
}  // namespace isg

using namespace isg;

extern "C" int ising_total_energy_noalloc(const ising_mesh* mc, int replica, const ising_params* p, double* e) {
    ising_mesh* m = const_cast<ising_mesh*>(mc);
    if (!m) return fail(ISING_ERR_ARG, "mesh is NULL");
    if (m->device < 0) return fail(ISING_ERR_ARG, "mesh was created without a device (device = -1)");
    if (replica < 0 || replica >= m->n_replicas) return fail(ISING_ERR_BOUNDS, "replica index out of range");
    if (!e) return fail(ISING_ERR_ARG, "e is NULL");
    int st = check_params(p);
    if (st != ISING_OK) return st;
    if ((st = mesh_settle(m)) != ISING_OK) return st;   // asynchronous spin transfers land first
    const int nb = energy_blocks_for(m->lat.natoms);
    if (nb > kNoAllocMaxBlocks)
        return fail(ISING_ERR_ARG, "replica too large: the allocation-free energy accepts at most 16777216 atoms "
                                   "(4096 blocks of 4096 sites)");
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != m->device) ISG_CUDA(cudaSetDevice(m->device));
    double* scratch = nullptr;
    st = scratch_for(m->device, &scratch);
    if (st == ISING_OK) {
        // stencil staged through the mesh's pinned host buffer (allocated with the mesh)
        Slot* hs = reinterpret_cast<Slot*>(m->h_pinned);
        int* hc = reinterpret_cast<int*>(hs + (size_t)kMaxSub * kMaxSlots);
        double* hout = m->h_pinned + (kScratchDoubles - 8);
        st = fill_query_stencil_host(m, *p, p->legacy_neighbours != 0, hs, hc);
        cudaError_t ce = cudaSuccess;
        if (st == ISING_OK)
            ce = cudaMemcpyAsync(m->d_slots, hs, sizeof(Slot) * kMaxSub * kMaxSlots, cudaMemcpyHostToDevice, m->stream);
        if (st == ISING_OK && ce == cudaSuccess)
            ce = cudaMemcpyAsync(m->d_slot_count, hc, sizeof(int) * kMaxSub, cudaMemcpyHostToDevice, m->stream);
        if (st == ISING_OK && ce == cudaSuccess) {
            ReduceLaunch a{};
            a.spins = m->d_spins + (int64_t)replica * 3 * m->lat.natoms;
            a.natoms = m->lat.natoms; a.nx = m->lat.nx; a.ny = m->lat.ny; a.nz = m->lat.nz; a.nsub = m->lat.nsub;
            a.n_rep = 1; a.ham = ham_of(*p); a.st = StencilDev{m->d_slots, m->d_slot_count, m->lat.nsub};
            a.layout = m->layout; a.block_tmp = scratch; a.out = scratch + kNoAllocMaxBlocks * 4;
            a.blocks_per_rep = nb;
            st = launch_energy_mag(a, m->stream);
        }
        if (st == ISING_OK && ce == cudaSuccess)
            ce = cudaMemcpyAsync(hout, scratch + kNoAllocMaxBlocks * 4, 4 * sizeof(double), cudaMemcpyDeviceToHost,
                                 m->stream);
        if (st == ISING_OK && ce == cudaSuccess) ce = cudaStreamSynchronize(m->stream);
        if (st == ISING_OK && ce != cudaSuccess) st = cuda_fail(ce, "allocation-free total energy");
        if (st == ISING_OK) *e = hout[0];
    }
    if (prev >= 0 && prev != m->device) cudaSetDevice(prev);
    return st;
}
