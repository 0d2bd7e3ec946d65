// exchange.cuh -- one replica-exchange round, executed by every thread of one block.
//
// Swap of temperature labels between neighbouring slots (the reference relabels
// TemperatureMeshArray and never moves spins, src/PT.f90:264-268).  Criterion
// min(1, exp((b_t - b_{t+1})(E_t - E_{t+1}))) with FP64 running energies.
// EVEN_ODD: all pairs (t, t+1) with t = round parity, in parallel (disjoint pairs).
// RANDOM_PAIRS: n sequential attempts at Index1 = nint(u (n-1)) (src/PT.f90:236-244).
//
// Global state is read with ld.global.cg and written with st.global.cg (L2 only): the
// persistent multi-ensemble engine runs this on whichever SM finishes a round last, so a
// line of this state left in an SM's L1 by an earlier round must never be read.
#pragma once
#include "internal.h"

namespace isg {

__device__ __forceinline__ void exchange_round(const ExchangeLaunch& a) {
    const int n = a.n;
    const uint32_t round = __ldcg(a.round);
    const uint2 key = philox_key(a.seed);
    const uint32_t tagw = (a.ensemble << 8) | kTagExchange;
    if (a.scheme == 0) {
        for (int t = (int)(round & 1u) + 2 * (int)threadIdx.x; t + 1 < n; t += 2 * (int)blockDim.x) {
            const uint4 r4 = philox4x32<10>(make_uint4((uint32_t)t, round, 0u, tagw), key);
            const int ra = __ldcg(a.t2r + t), rb = __ldcg(a.t2r + t + 1);
            const double d = (__ldcg(a.beta_t + t) - __ldcg(a.beta_t + t + 1)) * (__ldcg(&a.acc[ra].e) - __ldcg(&a.acc[rb].e));
            const double u = (double)(2u * (r4.x >> 9) + 1u) * (1.0 / 16777216.0);
            __stcg(a.stats + t, __ldcg(a.stats + t) + 1ull);
            if (d >= 0.0 || u < exp(d)) {
                __stcg(a.t2r + t, rb);
                __stcg(a.t2r + t + 1, ra);
                __stcg(a.stats + (n - 1) + t, __ldcg(a.stats + (n - 1) + t) + 1ull);
            }
        }
    } else if (threadIdx.x == 0) {
        for (int q = 0; q < n; ++q) {
            const uint4 r4 = philox4x32<10>(make_uint4((uint32_t)q, round, 1u, tagw), key);
            const double u0 = (double)(2u * (r4.x >> 9) + 1u) * (1.0 / 16777216.0);
            const double u1 = (double)(2u * (r4.y >> 9) + 1u) * (1.0 / 16777216.0);
            const double xv = u0 * (double)(n - 1);
            const int i1 = (int)(xv >= 0.0 ? floor(xv + 0.5) : -floor(-xv + 0.5));
            const int i2 = i1 == 0 ? 1 : (i1 == n - 1 ? n - 2 : i1 + 1);
            const int t = i1 < i2 ? i1 : i2;
            const int ra = __ldcg(a.t2r + t), rb = __ldcg(a.t2r + t + 1);
            const double d = (__ldcg(a.beta_t + t) - __ldcg(a.beta_t + t + 1)) * (__ldcg(&a.acc[ra].e) - __ldcg(&a.acc[rb].e));
            __stcg(a.stats + t, __ldcg(a.stats + t) + 1ull);
            if (d >= 0.0 || u1 < exp(d)) {
                __stcg(a.t2r + t, rb);
                __stcg(a.t2r + t + 1, ra);
                __stcg(a.stats + (n - 1) + t, __ldcg(a.stats + (n - 1) + t) + 1ull);
            }
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const int r = __ldcg(a.t2r + t);
        __stcg(a.r2t + r, t);
        __stcg(a.beta_rep + r, __ldcg(a.beta_t + t));
    }
    if (threadIdx.x == 0) __stcg(a.round, round + 1u);
}

}  // namespace isg
