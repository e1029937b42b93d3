// Plain delay-and-sum kernel: one launch per frame, one thread per voxel,
// tables and channel data read straight from global memory (the comparator
// for the fused kernel, and the one-frame path).
#pragma once

#include "das_common.cuh"

namespace rcabf {

// ------------------------------------------------------------------------
// Plain kernel: one launch per frame, one thread per voxel
// ------------------------------------------------------------------------
template <int IQ>
__device__ __forceinline__ float2 load_iq(const void *base, int64_t i)
{
    if constexpr (IQ == 0) return __ldg(reinterpret_cast<const float2 *>(base) + i);
    else if constexpr (IQ == 1) return __half22float2(reinterpret_cast<const __half2 *>(base)[i]);
    else if constexpr (IQ == 2) return __bfloat1622float2(reinterpret_cast<const __nv_bfloat162 *>(base)[i]);
    else {  // real RF, Q negated (RCA.m:476)
        const float2 v = __ldg(reinterpret_cast<const float2 *>(base) + i);
        return make_float2(v.x, -v.y);
    }
}

// PC: one output per receive element instead of the sum over them (the
// reference's no-sum kernel, NoSum/..._Nosum.cu:228-229, 275-278, 376-383):
// out[element][frame][tx][pix] = the element's term, 0 where it has none.
template <int MODE, int KIND, int IQ, bool PC>
__global__ void __launch_bounds__(256) plain_das_kernel(const __grid_constant__ PlainParams prm)
{
    using KT = KindTraits<KIND>;
    const DevGeom &g = prm.g;
    const int64_t n_vox = g.n_z * g.n_u * g.n_v;
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n_vox) return;
    const int64_t iz = v % g.n_z;
    const int64_t iu = (v / g.n_z) % g.n_u;
    const int64_t iv = v / (g.n_z * g.n_u);
    const int64_t rxkey = iu * g.n_z + iz, txkey = iv * g.n_z + iz;
    const int64_t n_rxkey = g.n_u * g.n_z, n_txkey = g.n_v * g.n_z;
    const int64_t pix = iz * g.s_z + iu * g.s_u + iv * g.s_v;
    float2 acc[1] = {make_float2(0.f, 0.f)};
    float2 acc_tx[1] = {make_float2(0.f, 0.f)};
    for (int tx = 0; tx < g.n_tx; ++tx) {
        const float4 t = __ldg(&g.tx_tab[(int64_t)tx * n_txkey + txkey]);
        bool cone_ok = ((MODE == MODE_EXACT) ? t.w : t.y) != 0.0f;
        if (g.cone_u != nullptr) cone_ok = cone_ok && g.cone_u[(int64_t)tx * n_rxkey + rxkey] != 0;
        if constexpr (PC) {
            if (!cone_ok) {   // masked: every element's term is 0
                for (int rx = 0; rx < g.n_ele; ++rx) {
                    float2 *o = prm.out + (((int64_t)rx * prm.n_frame + prm.frame) * g.n_tx + tx) * g.n_pix + pix;
                    if (!prm.accumulate) *o = make_float2(0.f, 0.f);
                }
            }
        }
        if (cone_ok) {
            const int64_t chan0 = (prm.frame * g.n_tx + tx) * (int64_t)g.n_ele;
            for (int rx = 0; rx < g.n_ele; ++rx) {
                const float4 e = __ldg(&g.rx_tab[(int64_t)rx * n_rxkey + rxkey]);
                const float ab = ab_value(g, tx, rx);
                Setup<KIND> st;
                if constexpr (MODE == MODE_EXACT)
                    setup_exact<KIND>(t, e, ab, ab_phasor(g, tx, rx), prm.n_sample, st);
                else
                    setup_ref<KIND>(t, e, ab, g.ref, prm.n_sample, st);
                if (!st.ok) {
                    if constexpr (PC) {
                        float2 *o = prm.out + (((int64_t)rx * prm.n_frame + prm.frame) * g.n_tx + tx) * g.n_pix + pix;
                        if (!prm.accumulate) *o = make_float2(0.f, 0.f);
                    }
                    continue;
                }
                const int64_t base = (chan0 + rx) * prm.n_sample + st.n0 - KT::LO;
                float2 tsum = make_float2(0.f, 0.f);
#pragma unroll
                for (int j = 0; j < KT::TAPS; ++j) {
                    const float2 x = load_iq<IQ>(prm.iq, base + j);
                    if constexpr (MODE == MODE_EXACT) {
                        tsum.x = fmaf(st.w[j], x.x, tsum.x);
                        tsum.y = fmaf(st.w[j], x.y, tsum.y);
                    } else if (j == 0) {
                        tsum = make_float2(__fmul_rn(st.w[0], x.x), __fmul_rn(st.w[0], x.y));
                    } else {
                        tsum.x = __fadd_rn(tsum.x, __fmul_rn(st.w[j], x.x));
                        tsum.y = __fadd_rn(tsum.y, __fmul_rn(st.w[j], x.y));
                    }
                }
                if constexpr (PC) {   // the element's own term, written as the reference's no-sum kernel does
                    float2 term;
                    if constexpr (MODE == MODE_EXACT) {
                        term.x = fmaf(st.P.x, tsum.x, -st.P.y * tsum.y);
                        term.y = fmaf(st.P.x, tsum.y, st.P.y * tsum.x);
                    } else {
                        const float cs = st.P.x, sn = st.P.y;
                        term.x = __fmul_rn(st.apod, __fadd_rn(__fmul_rn(tsum.x, cs), __fmul_rn(tsum.y, sn)));
                        term.y = __fmul_rn(st.apod, __fadd_rn(__fmul_rn(-tsum.x, sn), __fmul_rn(tsum.y, cs)));
                    }
                    float2 *o = prm.out + (((int64_t)rx * prm.n_frame + prm.frame) * g.n_tx + tx) * g.n_pix + pix;
                    if (prm.accumulate) { float2 q = *o; q.x += term.x; q.y += term.y; *o = q; }
                    else *o = term;
                    continue;
                }
                float2 &a = acc_tx[0];
                if constexpr (MODE == MODE_EXACT) {
                    a.x = fmaf(st.P.x, tsum.x, fmaf(-st.P.y, tsum.y, a.x));
                    a.y = fmaf(st.P.x, tsum.y, fmaf(st.P.y, tsum.x, a.y));
                } else {
                    const float cs = st.P.x, sn = st.P.y;
                    a.x = __fadd_rn(a.x, __fmul_rn(st.apod, __fadd_rn(__fmul_rn(tsum.x, cs), __fmul_rn(tsum.y, sn))));
                    a.y = __fadd_rn(a.y, __fmul_rn(st.apod, __fadd_rn(__fmul_rn(-tsum.x, sn), __fmul_rn(tsum.y, cs))));
                }
            }
        }
        if constexpr (PC) {
            acc_tx[0] = make_float2(0.f, 0.f);
            continue;
        }
        if (!prm.compound) {
            float2 *o = prm.out + (prm.frame * g.n_tx + tx) * g.n_pix + pix;
            if (prm.accumulate) { float2 q = *o; q.x += acc_tx[0].x; q.y += acc_tx[0].y; *o = q; }
            else *o = acc_tx[0];
        } else {
            acc[0].x = __fadd_rn(acc[0].x, acc_tx[0].x);
            acc[0].y = __fadd_rn(acc[0].y, acc_tx[0].y);
        }
        acc_tx[0] = make_float2(0.f, 0.f);
    }
    if (!PC && prm.compound) {
        float2 *o = prm.out + prm.frame * g.n_pix + pix;
        if (prm.accumulate) { float2 q = *o; q.x += acc[0].x; q.y += acc[0].y; *o = q; }
        else *o = acc[0];
    }
}

// Per-channel output (the reference's no-sum kernels) over all frames in one
// launch: one thread per (voxel, receive element), voxels fastest so that a
// warp's writes of one (element, frame, transmit) are contiguous; each
// (transmit, element) setup -- delays, weights, phasor, masks -- is formed
// once and serves every frame.  Per (voxel, element, transmit, frame) the
// arithmetic is the PC plain kernel's, in its order: the same bits, from one
// launch instead of one per frame.
template <int MODE, int KIND, int IQ>
__global__ void __launch_bounds__(256) pc_das_kernel(const __grid_constant__ PlainParams prm)
{
    using KT = KindTraits<KIND>;
    const DevGeom &g = prm.g;
    const int64_t n_vox = g.n_z * g.n_u * g.n_v;
    const int64_t n_rxkey = g.n_u * g.n_z, n_txkey = g.n_v * g.n_z;
    const int64_t n = n_vox * g.n_ele;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t v = i % n_vox;
        const int rx = (int)(i / n_vox);
        const int64_t iz = v % g.n_z;
        const int64_t iu = (v / g.n_z) % g.n_u;
        const int64_t iv = v / (g.n_z * g.n_u);
        const int64_t rxkey = iu * g.n_z + iz, txkey = iv * g.n_z + iz;
        const int64_t pix = iz * g.s_z + iu * g.s_u + iv * g.s_v;
        for (int tx = 0; tx < g.n_tx; ++tx) {
            const float4 t = __ldg(&g.tx_tab[(int64_t)tx * n_txkey + txkey]);
            bool ok = ((MODE == MODE_EXACT) ? t.w : t.y) != 0.0f;
            if (g.cone_u != nullptr) ok = ok && g.cone_u[(int64_t)tx * n_rxkey + rxkey] != 0;
            Setup<KIND> st;
            if (ok) {
                const float4 e = __ldg(&g.rx_tab[(int64_t)rx * n_rxkey + rxkey]);
                const float ab = ab_value(g, tx, rx);
                if constexpr (MODE == MODE_EXACT)
                    setup_exact<KIND>(t, e, ab, ab_phasor(g, tx, rx), prm.n_sample, st);
                else
                    setup_ref<KIND>(t, e, ab, g.ref, prm.n_sample, st);
                ok = st.ok;
            }
            for (int64_t f = 0; f < prm.n_frame; ++f) {
                float2 *o = prm.out + (((int64_t)rx * prm.n_frame + f) * g.n_tx + tx) * g.n_pix + pix;
                if (!ok) {
                    if (!prm.accumulate) *o = make_float2(0.f, 0.f);
                    continue;
                }
                const int64_t base = ((f * g.n_tx + tx) * (int64_t)g.n_ele + rx) * prm.n_sample + st.n0 - KT::LO;
                float2 tsum = make_float2(0.f, 0.f);
#pragma unroll
                for (int j = 0; j < KT::TAPS; ++j) {
                    const float2 x = load_iq<IQ>(prm.iq, base + j);
                    if constexpr (MODE == MODE_EXACT) {
                        tsum.x = fmaf(st.w[j], x.x, tsum.x);
                        tsum.y = fmaf(st.w[j], x.y, tsum.y);
                    } else if (j == 0) {
                        tsum = make_float2(__fmul_rn(st.w[0], x.x), __fmul_rn(st.w[0], x.y));
                    } else {
                        tsum.x = __fadd_rn(tsum.x, __fmul_rn(st.w[j], x.x));
                        tsum.y = __fadd_rn(tsum.y, __fmul_rn(st.w[j], x.y));
                    }
                }
                float2 term;
                if constexpr (MODE == MODE_EXACT) {
                    term.x = fmaf(st.P.x, tsum.x, -st.P.y * tsum.y);
                    term.y = fmaf(st.P.x, tsum.y, st.P.y * tsum.x);
                } else {
                    const float cs = st.P.x, sn = st.P.y;
                    term.x = __fmul_rn(st.apod, __fadd_rn(__fmul_rn(tsum.x, cs), __fmul_rn(tsum.y, sn)));
                    term.y = __fmul_rn(st.apod, __fadd_rn(__fmul_rn(-tsum.x, sn), __fmul_rn(tsum.y, cs)));
                }
                if (prm.accumulate) { float2 q = *o; q.x += term.x; q.y += term.y; *o = q; }
                else *o = term;
            }
        }
    }
}

}  // namespace rcabf
