// Delay-and-sum kernels for the RCA beamformer (sm_100a).
//
// Work unit: one voxel x one receive element x one transmit x one frame
// ("voxel.rx.tx.frame").  Per (voxel, rx, tx) the kernels form the sample
// index idx = Ttx(v, z) + Trx(u, z), the interpolation weights and the
// demodulation phasor ONCE, then reuse them for every frame the thread owns:
//     out[f] += P * sum_k w_k * s_f[n0 - LO + k]          (P = apod * phasor)
// which is the reference's per-frame expression (RCA.cu:307-380) with the
// frame-independent work hoisted out of the frame loop.
//
// fused_das_kernel: persistent CTAs walk (voxel tile, frame block) work items.
//   For every (tx, rx) step the CTA stages the sample window its tile needs --
//   rows [n_lo, n_hi] of the (tx, rx, frame block) slab, frames innermost --
//   into shared memory with cp.async (16-byte vectors, coalesced), triple
//   buffered so the copy of step s+2 overlaps the arithmetic of step s.
//   Each thread owns one voxel and FB frames; the sums over receive elements
//   and transmits stay in its registers.
// plain_das_kernel: one launch per frame, one thread per voxel, gathers
//   straight from the caller's layout in global memory.
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

// EXACT setup.  t = tx entry {itx, pr, pi, cone_v}, e = rx entry
// {irx, ar, ai, apod}, ab = aberration shift (samples), abp its phasor.
template <int KIND>
__device__ __forceinline__ void setup_exact(const float4 t, const float4 e, float ab, float2 abp,
                                            int n_sample, Setup<KIND> &s)
{
    using KT = KindTraits<KIND>;
    const float idx = __fadd_rn(__fadd_rn(t.x, e.x), ab);
    const float fl = floorf(idx);
    s.ok = (e.w > 0.0f) && (fl >= (float)KT::LO) && (fl < (float)(n_sample - 1 - KT::HI));
    s.n0 = s.ok ? (int)fl : 0;
    exact_weights<KIND>(idx - fl, s.w);
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

// ------------------------------------------------------------------------
// Fused persistent kernel
// ------------------------------------------------------------------------
template <int MODE, int KIND, int FB, int STORE>
__global__ void __launch_bounds__(FUSED_THREADS)
fused_das_kernel(const __grid_constant__ FusedParams prm)
{
    using T = typename StoreT<STORE>::T;
    using KT = KindTraits<KIND>;
    constexpr int ES = (int)sizeof(T);
    constexpr int ROWB = FB * ES;                  // bytes of one row in global memory
    constexpr int CS = ROWB < 16 ? ROWB : 16;      // cp.async chunk
    constexpr int CPR = ROWB / CS;                 // chunks per row
    constexpr bool TWO_LEVEL = (MODE == MODE_REF);

    extern __shared__ __align__(16) unsigned char smem[];
    const int tid = threadIdx.x;
    const int stage_bytes = prm.wmax * prm.row_words * 4;
    const int stride_s = prm.row_words * 4;
    {
        // The launch must provide FUSED_STAGES window buffers; if it did not,
        // record the error and touch nothing (uniform across the block).
        unsigned dyn;
        asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
        if (dyn < (unsigned)(FUSED_STAGES * stage_bytes) || stride_s < ROWB) {
            if (tid == 0) atomicAdd(prm.err_count, 1ull);
            return;
        }
    }

    for (int64_t item = blockIdx.x; item < prm.n_items; item += gridDim.x) {
        int ji = 0;
        while (ji + 1 < prm.n_jobs && prm.jobs[ji + 1].item_begin <= item) ++ji;
        const FusedJob &J = prm.jobs[ji];
        const DevGeom &g = J.g;
        const int lu = tid % J.tu;
        const int lv = (tid / J.tu) % J.tv;
        const int lz = tid / (J.tu * J.tv);
        const int64_t local = item - J.item_begin;
        const int64_t n_tiles = (int64_t)J.tiles_z * J.tiles_u * J.tiles_v;
        const int fb = (int)(local / n_tiles);
        const int64_t tile = local % n_tiles;
        const int tz = (int)(tile % J.tiles_z);
        const int tu = (int)((tile / J.tiles_z) % J.tiles_u);
        const int tv = (int)(tile / ((int64_t)J.tiles_z * J.tiles_u));
        const int64_t iz = (int64_t)tz * J.tz + lz;
        const int64_t iu = (int64_t)tu * J.tu + lu;
        const int64_t iv = (int64_t)tv * J.tv + lv;
        const bool vox = iz < g.n_z && iu < g.n_u && iv < g.n_v;
        const int64_t rxkey = iu * g.n_z + iz;
        const int64_t txkey = iv * g.n_z + iz;
        const int64_t n_rxkey = g.n_u * g.n_z;
        const int64_t n_txkey = g.n_v * g.n_z;
        const int n_steps = g.n_tx * g.n_ele;
        const char *S = reinterpret_cast<const char *>(J.S);

        float2 acc[FB], acc_tx[FB];
#pragma unroll
        for (int f = 0; f < FB; ++f) { acc[f] = make_float2(0.f, 0.f); acc_tx[f] = acc[f]; }

        auto slab = [&](int tx, int rx) -> const char * {
            return S + (((int64_t)tx * g.n_ele + rx) * J.n_fb + fb) * J.slab_bytes;
        };
        auto issue = [&](int s) {
            if (s < n_steps) {
                const int tx = s / g.n_ele, rx = s % g.n_ele;
                const Window w = step_window<MODE, KIND>(J, tx, rx, tu, tv, tz, ab_value(g, tx, rx), prm.wmax);
                if (!w.skip && !w.overflow) {
                    const char *src = slab(tx, rx) + (int64_t)w.lo * ROWB;
                    unsigned char *dst = smem + (s % FUSED_STAGES) * stage_bytes;
                    const int nch = w.count * CPR;
                    for (int c = tid; c < nch; c += FUSED_THREADS) {
                        const int r = c / CPR, q = c % CPR;
                        cp_async<CS>(dst + r * stride_s + q * CS, src + (int64_t)r * ROWB + q * CS);
                    }
                }
            }
            cp_async_commit();
        };

        // Prologue: stages 0 .. STAGES-2 in flight.
#pragma unroll
        for (int s = 0; s < FUSED_STAGES - 1; ++s) issue(s);

        float4 tcur = make_float4(0.f, 0.f, 0.f, 0.f);
        bool cone_ok = true;
        float4 enext = vox ? __ldg(&g.rx_tab[rxkey]) : make_float4(0.f, 0.f, 0.f, 0.f);

        for (int s = 0; s < n_steps; ++s) {
            const int tx = s / g.n_ele, rx = s % g.n_ele;
            cp_async_wait<FUSED_STAGES - 2>();
            __syncthreads();                       // step s landed; step s-1 buffer free
            issue(s + FUSED_STAGES - 1);

            const float4 e = enext;
            if (vox && s + 1 < n_steps) {
                const int rx1 = (s + 1) % g.n_ele;
                enext = __ldg(&g.rx_tab[(int64_t)rx1 * n_rxkey + rxkey]);
            }
            if (rx == 0 && vox) {
                tcur = __ldg(&g.tx_tab[(int64_t)tx * n_txkey + txkey]);
                const float cv = (MODE == MODE_EXACT) ? tcur.w : tcur.y;
                cone_ok = cv != 0.0f;
                if (g.cone_u != nullptr) cone_ok = cone_ok && g.cone_u[(int64_t)tx * n_rxkey + rxkey] != 0;
            }

            const float ab = ab_value(g, tx, rx);
            const Window w = step_window<MODE, KIND>(J, tx, rx, tu, tv, tz, ab, prm.wmax);
            if (!w.skip && vox && cone_ok) {
                Setup<KIND> st;
                if constexpr (MODE == MODE_EXACT)
                    setup_exact<KIND>(tcur, e, ab, ab_phasor(g, tx, rx), J.n_sample, st);
                else
                    setup_ref<KIND>(tcur, e, ab, g.ref, J.n_sample, st);
                if (st.ok) {
                    const int row0 = st.n0 - KT::LO - w.lo;
                    if (row0 < 0 || row0 + KT::TAPS > w.count) {
                        atomicAdd(prm.err_count, 1ull);   // never expected: window bound violated
                    } else if (!w.overflow) {
                        const char *rowp = reinterpret_cast<const char *>(smem) +
                                           (s % FUSED_STAGES) * stage_bytes + row0 * stride_s;
                        frame_loop<MODE, KIND, FB, STORE>(rowp, stride_s, st, TWO_LEVEL ? acc_tx : acc);
                    } else {
                        const char *rowp = slab(tx, rx) + (int64_t)(st.n0 - KT::LO) * ROWB;
                        frame_loop<MODE, KIND, FB, STORE>(rowp, ROWB, st, TWO_LEVEL ? acc_tx : acc);
                    }
                }
            }

            if (rx == g.n_ele - 1) {  // end of a transmit
                if (!J.compound && vox) {
                    const int64_t pix = iz * g.s_z + iu * g.s_u + iv * g.s_v;
                    float2 (&src)[FB] = TWO_LEVEL ? acc_tx : acc;
#pragma unroll
                    for (int f = 0; f < FB; ++f) {
                        const int fr = fb * FB + f;
                        if (fr < J.n_frame) {
                            float2 *o = J.out + ((int64_t)fr * g.n_tx + tx) * g.n_pix + pix;
                            if (J.accumulate) { float2 v = *o; v.x += src[f].x; v.y += src[f].y; *o = v; }
                            else *o = src[f];
                        }
                        src[f] = make_float2(0.f, 0.f);
                    }
                } else if (TWO_LEVEL) {
#pragma unroll
                    for (int f = 0; f < FB; ++f) {
                        acc[f].x = __fadd_rn(acc[f].x, acc_tx[f].x);
                        acc[f].y = __fadd_rn(acc[f].y, acc_tx[f].y);
                        acc_tx[f] = make_float2(0.f, 0.f);
                    }
                }
            }
        }
        cp_async_wait<0>();
        __syncthreads();  // all buffers idle before the next work item reuses them

        if (J.compound && vox) {
            const int64_t pix = iz * g.s_z + iu * g.s_u + iv * g.s_v;
#pragma unroll
            for (int f = 0; f < FB; ++f) {
                const int fr = fb * FB + f;
                if (fr < J.n_frame) {
                    float2 *o = J.out + (int64_t)fr * g.n_pix + pix;
                    if (J.accumulate) { float2 v = *o; v.x += acc[f].x; v.y += acc[f].y; *o = v; }
                    else *o = acc[f];
                }
            }
        }
    }
}

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

template <int MODE, int KIND, int IQ>
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
                if (!st.ok) continue;
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
    if (prm.compound) {
        float2 *o = prm.out + prm.frame * g.n_pix + pix;
        if (prm.accumulate) { float2 q = *o; q.x += acc[0].x; q.y += acc[0].y; *o = q; }
        else *o = acc[0];
    }
}

}  // namespace rcabf
