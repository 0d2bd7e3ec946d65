// winding.cuh -- the Berg-Luscher solid-angle term shared by the winding kernels.
#pragma once
#include <cstdint>

namespace isg {

// arc_winding (rsp:284-318): 2*atan2(Im, Re) of
// (1 + s1.s2 + s2.s3 + s3.s1 + i s1.(s2 x s3)) / sqrt(2(1+s1.s2)(1+s2.s3)(1+s3.s1)).
template <typename T>
__device__ __forceinline__ T arc_winding_t(const T* s1, const T* s2, const T* s3) {
    const T d12 = s1[0] * s2[0] + s1[1] * s2[1] + s1[2] * s2[2];
    const T d23 = s2[0] * s3[0] + s2[1] * s3[1] + s2[2] * s3[2];
    const T d31 = s3[0] * s1[0] + s3[1] * s1[1] + s3[2] * s1[2];
    const T cx = s2[1] * s3[2] - s2[2] * s3[1];
    const T cy = s2[2] * s3[0] - s2[0] * s3[2];
    const T cz = s2[0] * s3[1] - s2[1] * s3[0];
    T re = T(1) + d12 + d23 + d31;
    T im = s1[0] * cx + s1[1] * cy + s1[2] * cz;
    const T nrm = sqrt(T(2) * (T(1) + d12) * (T(1) + d23) * (T(1) + d31));
    re = re / nrm;
    im = im / nrm;
    return T(2) * atan2(im, re);
}

template <typename T>
__device__ __forceinline__ void load_unit(const float* sx, const float* sy, const float* sz, int64_t j, T* o) {
    const T x = (T)sx[j], y = (T)sy[j], z = (T)sz[j];
    const T n = sqrt(x * x + y * y + z * z);
    o[0] = x / n; o[1] = y / n; o[2] = z / n;
}

}  // namespace isg
