// ensembles.cu -- launch of the persistent multi-ensemble engine (ensembles_kernel.cuh).
#include <cudaTypedefs.h>

#include <algorithm>

#include "ensembles.h"

namespace isg {

static const void* ens_kernel(int move, int dmi, bool hk, int loader) {
    // kind 0 (no DMI) runs the bulk form with D = 0: h gains 0 * (...) terms only
    if (dmi == 0) dmi = 1;
    return move == 0 ? ensembles_kernel_uniform(dmi, hk, loader) : ensembles_kernel_ball(dmi, hk, loader);
}

// Dynamic shared memory of a launch: the staged ring, or the fused kernel's row slots.
static size_t ens_smem(int loader, size_t fused_smem) {
    return loader == 1 ? (size_t)kStSmemBytes : (loader == 2 ? fused_smem : 0);
}

// The staged and fused kernels' shared-memory limit is a per-device attribute.  It is raised
// where a schedule is applied (ensembles_blocks_per_sm, on the engine's device and outside
// any stream capture), before the first launch of that schedule.
static int ens_smem_attr(const void* fn, int loader, size_t smem) {
    if (loader != 0) ISG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    return ISING_OK;
}

static int ens_threads(int loader, int threads) { return loader == 1 ? kStThreads : threads; }

int ensembles_blocks_per_sm(int move, int dmi, bool has_k, int loader, int threads, size_t smem, int* out) {
    const void* fn = ens_kernel(move, dmi, has_k, loader);
    const size_t sb = ens_smem(loader, smem);
    const int st = ens_smem_attr(fn, loader, sb);
    if (st != ISING_OK) return st;
    int n = 0;
    ISG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, ens_threads(loader, threads), sb));
    *out = n;
    return ISING_OK;
}

int launch_ensembles(const EnsParams& P, int move, int dmi, bool has_k, int loader, int threads, int grid,
                     size_t smem, cudaStream_t s) {
    const int maxt = loader == 2 ? kFuMaxThreads : kEnsMaxThreads;
    if (threads < 32 || threads > maxt || threads % 32) return fail(ISING_ERR_ARG, "block size out of range for the loader");
    if (loader == 1 && threads != kStSub * kStG * 32) return fail(ISING_ERR_ARG, "the staged loader runs 256-thread blocks");
    if (P.n_ens < 1 || P.n_ens > kMaxEnsembles) return fail(ISING_ERR_ARG, "1..16 ensembles per engine");
    const void* fn = ens_kernel(move, dmi, has_k, loader);
    void* args[] = {const_cast<EnsParams*>(&P)};
    // staged: the schedule's 256 compute threads plus the copy warp
    ISG_CUDA(cudaLaunchKernel(fn, dim3(grid), dim3(ens_threads(loader, threads)), args, ens_smem(loader, smem), s));
    return ISING_OK;
}

bool ensembles_encode_maps(float* spins, int nx, int ny, int n_rep, EnsMaps* m) {
    auto enc = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(tensor_map_encoder());
    if (!enc) return false;
    // (entry, y, x, colour, 3 replica + component) of W = 64 entries per packed row
    const cuuint64_t half = (cuuint64_t)nx * ny * 64;
    const cuuint64_t dims[5] = {64, (cuuint64_t)ny, (cuuint64_t)nx, 2, 3 * (cuuint64_t)n_rep};
    const cuuint64_t strides[4] = {64 * 4, (cuuint64_t)ny * 64 * 4, half * 4, 2 * half * 4};
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    // with nx < kStG + 2 every plane group wraps and the next map is never used
    const cuuint32_t nb = (cuuint32_t)std::min(kStG + 2, nx);
    const cuuint32_t boxes[4][5] = {{64, 1, nb, 1, 3}, {64, 1, kStG, 1, 3}, {64, 1, kStG, 1, 1}, {64, 1, 1, 1, 1}};
    CUtensorMap* out[4] = {&m->next, &m->own, &m->ctr, &m->halo};
    for (int i = 0; i < 4; ++i)
        if (enc(out[i], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, spins, dims, strides, boxes[i], es,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    return true;
}

}  // namespace isg
