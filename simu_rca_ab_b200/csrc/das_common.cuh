// Device code shared by the delay-and-sum kernels of the RCA beamformer
// (sm_100a): sample conversion, interpolation weights, the per
// (voxel, rx, tx) setup, the frame loop, cp.async helpers and the per-step
// sample window of a voxel tile.
//
// Work unit: one voxel x one receive element x one transmit x one frame
// ("voxel.rx.tx.frame").  Per (voxel, rx, tx) the kernels form the sample
// index idx = Ttx(v, z) + Trx(u, z), the interpolation weights and the
// demodulation phasor ONCE, then reuse them for every frame the thread owns:
//     out[f] += P * sum_k w_k * s_f[n0 - LO + k]          (P = apod * phasor)
// which is the reference's per-frame expression (RCA.cu:307-380) with the
// frame-independent work hoisted out of the frame loop.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "rcabf_internal.h"

namespace rcabf {

#define RCABF_PI_F 3.14159265358979323846f

// ------------------------------------------------------------------------
// Sample conversion
// ------------------------------------------------------------------------
template <int STORE> struct StoreT;
template <> struct StoreT<ST_F32>  { using T = float2; };
template <> struct StoreT<ST_F16>  { using T = __half2; };
template <> struct StoreT<ST_BF16> { using T = __nv_bfloat162; };

__device__ __forceinline__ float2 to_f2(const float2 v) { return v; }
__device__ __forceinline__ float2 to_f2(const __half2 v) { return __half22float2(v); }
__device__ __forceinline__ float2 to_f2(const __nv_bfloat162 v) { return __bfloat1622float2(v); }

// Loads N consecutive samples (N * sizeof(T) in {4, 8, 16} bytes) with one
// vector instruction.
template <typename T, int N>
__device__ __forceinline__ void load_vec(const T *p, T (&v)[N])
{
    constexpr int B = N * (int)sizeof(T);
    static_assert(B == 4 || B == 8 || B == 16, "vector width");
    if constexpr (B == 16) {
        uint4 r = *reinterpret_cast<const uint4 *>(p);
        memcpy(v, &r, 16);
    } else if constexpr (B == 8) {
        uint2 r = *reinterpret_cast<const uint2 *>(p);
        memcpy(v, &r, 8);
    } else {
        uint32_t r = *reinterpret_cast<const uint32_t *>(p);
        memcpy(v, &r, 4);
    }
}

// ------------------------------------------------------------------------
// Interpolation weights, EXACT mode
// ------------------------------------------------------------------------
// cos / sin of pi * k / 12 for k = 0..23 (all the angles pi*o/W with
// W in {2, 3, 4} fall on this grid).
__device__ __forceinline__ float cos_pi12(int k)
{
    const float t[24] = {1.0f, 0.96592582628906831f, 0.86602540378443865f, 0.70710678118654752f,
                         0.5f, 0.25881904510252076f, 0.0f, -0.25881904510252076f,
                         -0.5f, -0.70710678118654752f, -0.86602540378443865f, -0.96592582628906831f,
                         -1.0f, -0.96592582628906831f, -0.86602540378443865f, -0.70710678118654752f,
                         -0.5f, -0.25881904510252076f, 0.0f, 0.25881904510252076f,
                         0.5f, 0.70710678118654752f, 0.86602540378443865f, 0.96592582628906831f};
    return t[((k % 24) + 24) % 24];
}

// Weights w_j for taps on samples n0 - LO + j, fractional offset d in [0, 1).
// Kernel sinc(x) * sinc(x / W) at x_j = d + LO - j, written as
//   W sin(pi x) sin(pi x / W) / (pi^2 x^2),
// with sin(pi (d + o)) = (-1)^o sin(pi d) and
//      sin(pi (d + o) / W) = sin(pi d / W) cos(pi o / W) + cos(pi d / W) sin(pi o / W),
// so one sinpif and one sincospif serve all taps.
template <int KIND>
__device__ __forceinline__ void exact_weights(float d, float (&w)[KindTraits<KIND>::TAPS])
{
    using KT = KindTraits<KIND>;
    if constexpr (KIND == K_QUAD3) {
        // Lagrange quadratic through n0-1, n0, n0+1 (RCA.cu:355-357).
        w[0] = 0.5f * d * (d - 1.0f);
        w[1] = (1.0f - d) * (1.0f + d);
        w[2] = 0.5f * d * (d + 1.0f);
    } else {
        constexpr int W = KT::WIN;
        const float s1 = sinpif(d);
        float sa, ca;
        sincospif(d * (1.0f / (float)W), &sa, &ca);
        const float A = s1 * ((float)W / (RCABF_PI_F * RCABF_PI_F));
#pragma unroll
        for (int j = 0; j < KT::TAPS; ++j) {
            const int o = KT::LO - j;
            const float x = d + (float)o;
            const float cw = cos_pi12(o * (12 / W));
            const float sw = cos_pi12(o * (12 / W) - 6);  // sin(t) = cos(t - pi/2)
            const float sinw = fmaf(sa, cw, ca * sw);
            const float num = ((o & 1) ? -A : A) * sinw;
            w[j] = __fdividef(num, x * x);
        }
        if (d == 0.0f) {
#pragma unroll
            for (int j = 0; j < KT::TAPS; ++j) w[j] = (j == KT::LO) ? 1.0f : 0.0f;
        }
    }
}

// ------------------------------------------------------------------------
// Interpolation weights and phase, REF_COMPAT mode: the reference kernel's
// single-precision expressions, operation for operation, with every
// rounding explicit (this code is compiled with -fmad=false as well).
// ------------------------------------------------------------------------
__device__ __forceinline__ float ref_sinc(float x)  // RCA.cu:79-82
{
    return fminf(fdividef(sinpif(x), __fmul_rn(RCABF_PI_F, x)), 1.0f);
}

template <int KIND>
__device__ __forceinline__ void ref_weights(float d, float (&w)[KindTraits<KIND>::TAPS])
{
    static_assert(KIND == K_QUAD3 || KIND == K_REF6, "reference kernels only");
    if constexpr (KIND == K_REF6) {  // RCA.cu:331-336
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            const float x = __fadd_rn(d, (float)(2 - j));
            w[j] = __fmul_rn(ref_sinc(x), ref_sinc(__fdiv_rn(x, 2.0f)));
        }
    } else {  // RCA.cu:355-357
        const float dm1 = __fsub_rn(d, 1.0f), dp1 = __fadd_rn(d, 1.0f);
        w[0] = __fdiv_rn(__fmul_rn(d, dm1), 2.0f);
        w[1] = __fmul_rn(-dm1, dp1);
        w[2] = __fdiv_rn(__fmul_rn(d, dp1), 2.0f);
    }
}

// Per (voxel, rx, tx) setup result.
template <int KIND>
struct Setup {
    float w[KindTraits<KIND>::TAPS];
    float2 P;      // EXACT: apod * phasor.  REF: (cos, sin) of the phase
    float apod;    // REF only
    int n0;
    bool ok;
};

// Polyphase weight table (EXACT mode, windowed-sinc kernels): for phase
// q = 0..WT_Q-1, row q holds the TAPS weights at d = q / WT_Q (padded to 8)
// followed by their increments to d = (q + 1) / WT_Q, built in FP64 on the
// host.  Linear interpolation between phases leaves an error below
// (1/WT_Q)^2 / 8 * max|k''| ~ 1e-5 of a weight, far under the FP32 sum's.
constexpr int WT_Q = 256;
constexpr int WT_ROW = 16;                               // floats per phase
constexpr int WT_BYTES = WT_Q * WT_ROW * 4;

template <int MODE, int KIND>
struct UsesTable { static constexpr bool value = (MODE == MODE_EXACT) && (KIND != K_QUAD3); };

template <int KIND>
__device__ __forceinline__ void table_weights(const float *wt, float d, float (&w)[KindTraits<KIND>::TAPS])
{
    constexpr int TAPS = KindTraits<KIND>::TAPS;
    const float x = d * (float)WT_Q;
    const int q = min((int)x, WT_Q - 1);
    const float f = x - (float)q;
    const float4 *p = reinterpret_cast<const float4 *>(wt + q * WT_ROW);
    const float4 a0 = p[0], b0 = p[2];
    const float wa[4] = {a0.x, a0.y, a0.z, a0.w}, wb[4] = {b0.x, b0.y, b0.z, b0.w};
#pragma unroll
    for (int j = 0; j < (TAPS < 4 ? TAPS : 4); ++j) w[j] = fmaf(f, wb[j], wa[j]);
    if constexpr (TAPS > 4) {
        const float4 a1 = p[1], b1 = p[3];
        const float wc[4] = {a1.x, a1.y, a1.z, a1.w}, wd[4] = {b1.x, b1.y, b1.z, b1.w};
#pragma unroll
        for (int j = 4; j < TAPS; ++j) w[j] = fmaf(f, wd[j - 4], wc[j - 4]);
    }
}

// EXACT setup.  t = tx entry {itx, pr, pi, cone_v}, e = rx entry
// {irx, ar, ai, apod}, ab = aberration shift (samples), abp its phasor.
// wt = shared-memory polyphase table, or NULL to evaluate the kernel directly.
template <int KIND>
__device__ __forceinline__ void setup_exact(const float4 t, const float4 e, float ab, float2 abp,
                                            int n_sample, Setup<KIND> &s, const float *wt = nullptr)
{
    using KT = KindTraits<KIND>;
    const float idx = __fadd_rn(__fadd_rn(t.x, e.x), ab);
    const float fl = floorf(idx);
    s.ok = (e.w > 0.0f) && (fl >= (float)KT::LO) && (fl < (float)(n_sample - 1 - KT::HI));
    s.n0 = s.ok ? (int)fl : 0;
    if (KIND != K_QUAD3 && wt != nullptr) table_weights<KIND>(wt, idx - fl, s.w);
    else exact_weights<KIND>(idx - fl, s.w);
    // P = (pr + j pi) (ar + j ai) (abr + j abi)
    float2 q = make_float2(fmaf(t.y, e.y, -t.z * e.z), fmaf(t.y, e.z, t.z * e.y));
    s.P = make_float2(fmaf(q.x, abp.x, -q.y * abp.y), fmaf(q.x, abp.y, q.y * abp.x));
    s.apod = e.w;
}

// REF_COMPAT setup.  t = {delay_tx, cone_v, z, 0}, e = {delay_rx, apod, valid, 0},
// ab = aberration delay (s).  RCA.cu:308-323, 371-373.
template <int KIND>
__device__ __forceinline__ void setup_ref(const float4 t, const float4 e, float ab,
                                          const RefScalars &rs, int n_sample, Setup<KIND> &s)
{
    using KT = KindTraits<KIND>;
    const float drx = __fadd_rn(ab, e.x);
    const float idx = __fmul_rn(__fadd_rn(__fadd_rn(t.x, drx), rs.t0), rs.fs);
    const int n0 = (int)floorf(idx);
    s.ok = (e.z != 0.0f) && (n0 >= KT::LO) && (n0 < n_sample - 1 - KT::HI);
    s.n0 = s.ok ? n0 : 0;
    ref_weights<KIND>(__fsub_rn(idx, (float)n0), s.w);
    const float delta = __fadd_rn(
        __fmul_rn(__fmul_rn(__fmul_rn(-2.0f, RCABF_PI_F), idx), rs.ratio),
        __fmul_rn(__fmul_rn(__fmul_rn(__fmul_rn(4.0f, RCABF_PI_F), rs.fd), t.z), rs.inv_c));
    s.P = make_float2(cosf(delta), sinf(delta));
    s.apod = e.y;
}

// ------------------------------------------------------------------------
// Frame loop: acc[f] += P * sum_j w_j s_f[row j]
// rowp points at tap 0 of frame 0; rows are `stride` bytes apart, frames
// are consecutive samples within a row.
// ------------------------------------------------------------------------
template <int MODE, int KIND, int FB, int STORE>
__device__ __forceinline__ void frame_loop(const char *rowp, int stride, const Setup<KIND> &s,
                                           float2 (&acc)[FB])
{
    using T = typename StoreT<STORE>::T;
    constexpr int TAPS = KindTraits<KIND>::TAPS;
    constexpr int VMAX = 16 / (int)sizeof(T);
    constexpr int VEC = FB < VMAX ? FB : VMAX;
#pragma unroll
    for (int c = 0; c < FB; c += VEC) {
        float2 tsum[VEC];
#pragma unroll
        for (int j = 0; j < TAPS; ++j) {
            T raw[VEC];
            load_vec<T, VEC>(reinterpret_cast<const T *>(rowp + j * stride) + c, raw);
#pragma unroll
            for (int v = 0; v < VEC; ++v) {
                const float2 x = to_f2(raw[v]);
                if constexpr (MODE == MODE_EXACT) {
                    if (j == 0) {
                        tsum[v] = make_float2(s.w[0] * x.x, s.w[0] * x.y);
                    } else {
                        tsum[v].x = fmaf(s.w[j], x.x, tsum[v].x);
                        tsum[v].y = fmaf(s.w[j], x.y, tsum[v].y);
                    }
                } else {
                    if (j == 0) {
                        tsum[v] = make_float2(__fmul_rn(s.w[0], x.x), __fmul_rn(s.w[0], x.y));
                    } else {
                        tsum[v].x = __fadd_rn(tsum[v].x, __fmul_rn(s.w[j], x.x));
                        tsum[v].y = __fadd_rn(tsum[v].y, __fmul_rn(s.w[j], x.y));
                    }
                }
            }
        }
#pragma unroll
        for (int v = 0; v < VEC; ++v) {
            float2 &a = acc[c + v];
            const float2 t = tsum[v];
            if constexpr (MODE == MODE_EXACT) {
                a.x = fmaf(s.P.x, t.x, fmaf(-s.P.y, t.y, a.x));
                a.y = fmaf(s.P.x, t.y, fmaf(s.P.y, t.x, a.y));
            } else {  // RCA.cu:375-380
                const float cs = s.P.x, sn = s.P.y;
                a.x = __fadd_rn(a.x, __fmul_rn(s.apod, __fadd_rn(__fmul_rn(t.x, cs), __fmul_rn(t.y, sn))));
                a.y = __fadd_rn(a.y, __fmul_rn(s.apod, __fadd_rn(__fmul_rn(-t.x, sn), __fmul_rn(t.y, cs))));
            }
        }
    }
}

// ------------------------------------------------------------------------
// cp.async helpers (sm_80+ asynchronous global -> shared copies)
// ------------------------------------------------------------------------
template <int BYTES>
__device__ __forceinline__ void cp_async(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
    else if constexpr (BYTES == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// ------------------------------------------------------------------------
// Window of sample rows a tile needs for one (tx, rx) step
// ------------------------------------------------------------------------
struct Window {
    int lo, count;
    bool skip, overflow;
};

// Rows [lo, lo + count) of the (tx, rx) slab hold every tap any voxel of
// the tile can use in this step; windows longer than `wmax` rows (the
// staging capacity) are read from global memory instead.
template <int MODE, int KIND>
__device__ __forceinline__ Window step_window(const FusedJob &J, int tx, int rx, int tu, int tv, int tz,
                                              float ab, int wmax)
{
    using KT = KindTraits<KIND>;
    Window w;
    w.lo = 0; w.count = 0; w.overflow = false; w.skip = true;
    const float2 rr = J.rx_range[((int64_t)rx * J.tiles_u + tu) * J.tiles_z + tz];
    const float2 tr = J.tx_range[((int64_t)tx * J.tiles_v + tv) * J.tiles_z + tz];
    if (!(rr.x <= rr.y) || !(tr.x <= tr.y)) return w;
    float lo_f, hi_f;
    if constexpr (MODE == MODE_EXACT) {
        lo_f = __fadd_rn(__fadd_rn(tr.x, rr.x), ab);
        hi_f = __fadd_rn(__fadd_rn(tr.y, rr.y), ab);
    } else {
        const RefScalars &rs = J.g.ref;
        lo_f = __fmul_rn(__fadd_rn(__fadd_rn(tr.x, __fadd_rn(ab, rr.x)), rs.t0), rs.fs);
        hi_f = __fmul_rn(__fadd_rn(__fadd_rn(tr.y, __fadd_rn(ab, rr.y)), rs.t0), rs.fs);
    }
    // Usable n0 lie in [LO, n_sample - 2 - HI]; rows touched in [0, n_sample - 2].
    const float fmax_n = (float)(J.n_sample);
    lo_f = fminf(fmaxf(floorf(lo_f), -1.0f), fmax_n);
    hi_f = fminf(fmaxf(floorf(hi_f), -1.0f), fmax_n);
    int lo = (int)lo_f - KT::LO;
    int hi = (int)hi_f - KT::LO + KT::TAPS - 1;
    lo = max(lo, 0);
    hi = min(hi, J.n_sample - 2);
    if (hi < lo) return w;
    w.skip = false;
    w.lo = lo;
    w.count = hi - lo + 1;
    w.overflow = w.count > wmax;
    return w;
}

__device__ __forceinline__ float ab_value(const DevGeom &g, int tx, int rx)
{
    if (g.ab == nullptr) return 0.0f;
    return g.ab[g.ab_per_tx ? (int64_t)tx * g.n_ele + rx : rx];
}
__device__ __forceinline__ float2 ab_phasor(const DevGeom &g, int tx, int rx)
{
    if (g.ab_ph == nullptr) return make_float2(1.0f, 0.0f);
    return g.ab_ph[g.ab_per_tx ? (int64_t)tx * g.n_ele + rx : rx];
}


}  // namespace rcabf
