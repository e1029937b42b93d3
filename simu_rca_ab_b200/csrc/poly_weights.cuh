// Interpolation weights from the fitted polynomials of weight_poly.h, shared
// by the voxel-blocked SIMT kernel and the tensor-core kernel.
#pragma once

#include "das_common.cuh"
#include "weight_poly.h"

namespace rcabf {

// Weights w[0..TAPS) at fractional offset d in [0, 1), from the degree-DEG
// polynomials.
template <int KIND, int DEG>
__device__ __forceinline__ void poly_weights(float d, float (&w)[KindTraits<KIND>::TAPS])
{
    if constexpr (KIND == K_QUAD3) {
        w[0] = 0.5f * d * (d - 1.0f);
        w[1] = (1.0f - d) * (1.0f + d);
        w[2] = 0.5f * d * (d + 1.0f);
    } else {
        // w_j(u) = E_j(u^2) + u O_j(u^2) and w_{T-1-j}(u) = w_j(-u) = E_j - u O_j:
        // both weights of a mirrored pair from one even and one odd Horner
        // chain in s = u^2 (DEG + 1 FMAs per pair)
        using WP = WeightPoly<KIND, DEG>;
        constexpr int T = KindTraits<KIND>::TAPS;
        static_assert(DEG % 2 == 0, "even degree");
        const float u = fmaf(2.0f, d, -1.0f);
        const float s = u * u;
#pragma unroll
        for (int j = 0; j < WP::HALF; ++j) {
            float e = WP::c(j, DEG);
#pragma unroll
            for (int m = DEG - 2; m >= 0; m -= 2) e = fmaf(e, s, WP::c(j, m));
            float o = WP::c(j, DEG - 1);
#pragma unroll
            for (int m = DEG - 3; m >= 1; m -= 2) o = fmaf(o, s, WP::c(j, m));
            w[j] = fmaf(u, o, e);             // w_j(d)
            w[T - 1 - j] = fmaf(-u, o, e);    // w_{T-1-j}(d) = w_j(1 - d)
        }
    }
}

}  // namespace rcabf
