// ensembles_uniform.cu -- persistent-engine kernels for the uniform unit-vector move
// (one translation unit per move kind, so the variants compile in parallel).
#include "ensembles_kernel.cuh"

namespace isg {

template <int D, bool K>
static const void* fn() { return reinterpret_cast<const void*>(&k_ensembles<0, D, K>); }

const void* ensembles_kernel_uniform(int dmi, bool has_k) {
    switch (dmi) {
        case 1: return has_k ? fn<1, true>() : fn<1, false>();
        case 2: return has_k ? fn<2, true>() : fn<2, false>();
        default: return has_k ? fn<3, true>() : fn<3, false>();
    }
}

}  // namespace isg
