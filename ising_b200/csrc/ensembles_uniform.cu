// ensembles_uniform.cu -- persistent-engine kernels for the uniform unit-vector move
// (one translation unit per move kind, so the variants compile in parallel).
#include "ensembles_kernel.cuh"

namespace isg {

template <int D, bool K>
static const void* fn(bool staged) {
    return staged ? reinterpret_cast<const void*>(&k_ensembles<0, D, K, true>)
                  : reinterpret_cast<const void*>(&k_ensembles<0, D, K, false>);
}

const void* ensembles_kernel_uniform(int dmi, bool has_k, bool staged) {
    switch (dmi) {
        case 1: return has_k ? fn<1, true>(staged) : fn<1, false>(staged);
        case 2: return has_k ? fn<2, true>(staged) : fn<2, false>(staged);
        default: return has_k ? fn<3, true>(staged) : fn<3, false>(staged);
    }
}

}  // namespace isg
