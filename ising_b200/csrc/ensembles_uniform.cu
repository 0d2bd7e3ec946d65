// ensembles_uniform.cu -- persistent-engine kernels for the uniform unit-vector move
// (one translation unit per move kind, so the variants compile in parallel).
#include "ensembles_fused.cuh"

namespace isg {

template <int D, bool K>
static const void* fn(int loader) {
    if (loader == 2) return reinterpret_cast<const void*>(&k_ensembles_fused<0, D, K>);
    return loader == 1 ? reinterpret_cast<const void*>(&k_ensembles<0, D, K, true>)
                       : reinterpret_cast<const void*>(&k_ensembles<0, D, K, false>);
}

const void* ensembles_kernel_uniform(int dmi, bool has_k, int loader) {
    switch (dmi) {
        case 1: return has_k ? fn<1, true>(loader) : fn<1, false>(loader);
        case 2: return has_k ? fn<2, true>(loader) : fn<2, false>(loader);
        default: return has_k ? fn<3, true>(loader) : fn<3, false>(loader);
    }
}

}  // namespace isg
