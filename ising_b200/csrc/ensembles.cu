// ensembles.cu -- launch of the persistent multi-ensemble engine (ensembles_kernel.cuh).
#include "ensembles.h"

namespace isg {

static const void* ens_kernel(int move, int dmi, bool hk) {
    // kind 0 (no DMI) runs the bulk form with D = 0: h gains 0 * (...) terms only
    if (dmi == 0) dmi = 1;
    return move == 0 ? ensembles_kernel_uniform(dmi, hk) : ensembles_kernel_ball(dmi, hk);
}

int ensembles_blocks_per_sm(int move, int dmi, bool has_k, int threads, int* out) {
    int n = 0;
    ISG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ens_kernel(move, dmi, has_k), threads, 0));
    *out = n;
    return ISING_OK;
}

int launch_ensembles(const EnsParams& P, int move, int dmi, bool has_k, int threads, int grid, cudaStream_t s) {
    if (threads < 32 || threads > kEnsMaxThreads || threads % 32)
        return fail(ISING_ERR_ARG, "block size must be 32..256, whole warps");
    if (P.n_ens < 1 || P.n_ens > kMaxEnsembles) return fail(ISING_ERR_ARG, "1..16 ensembles per engine");
    void* args[] = {const_cast<EnsParams*>(&P)};
    ISG_CUDA(cudaLaunchKernel(ens_kernel(move, dmi, has_k), dim3(grid), dim3(threads), args, 0, s));
    return ISING_OK;
}

}  // namespace isg
