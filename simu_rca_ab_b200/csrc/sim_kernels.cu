// Frequency-domain ultrasound simulator (the upstream producer of channel
// data): the field one transducer element radiates to (or receives from) one
// scatterer at one frequency, for every (frequency, scatterer, element).
//
// Linear acoustic model (SIMUS, Garcia 2022) as the reference simulator uses
// it (MATLAB/lib/simulator/SimUS_CUDARCA.cu:83-206, 209-379):
//   E(f, s, e) = sum over sub-elements of
//                G(r, k) * D_az(az, k) * D_el(r, el, k) * exp(i w lens)
//   G(r, k)    = exp(i k r) / r                       (k complex: attenuation)
//   D_az       = sinc(k w sin(az) / 2) [* cos(az) with a baffle]
//                (main lobe only: 0 once |argument| >= pi)
//   D_el       = D_az's form at the elevation angle with the element width
//                when the elevation focus is beyond 10 m, else the 4-term
//                multi-Gaussian beam of a focused element of height h,
//                sum_g A_g sqrt(pi / a_g) exp(b^2 / (4 a_g) + c),
//                a_g = B_g / h^2 + i k (r - F) / (2 r F), b = -i k y / r,
//                c = i k y^2 / (2 r), y = r sin(el)
// with r, az = asin((xs - xe) / r) - az_e, el = asin((ys - ye) / r) - el_e.
// The reference evaluates these per (frequency, scatterer, transmit) inside
// its transmit kernel, once for every transmit; here they are evaluated once
// per (frequency, scatterer, element) and every transmit of a group of
// events that share scatterer positions takes its delay / apodisation
// weight from the same value (the transmit field is linear in them), which
// removes the transmit count from the transcendental work.
//
// Kernels:
//   element_field_kernel  E(f, s, e) into memory (rcabf_sim_element_field)
//   sim_tx_kernel         TX(f, s, g) = T(f) b(s, g) sum_e E_tx(f, s, e) a(e, g) e^{i w d(e, g)}
//                         (rcabf_sim_tx_field; SimUS_CUDARCA.cu:209-292, SimUS_CUDARCA.m:319-344)
//   sim_rx_kernel         S(f, e', g) = R(f) a'(e', g) sum_s E_rx(f, s, e') TX(f, s, g)
//                         (rcabf_sim_rx_spectrum; SimUS_CUDARCA.cu:294-379, SimUS_CUDARCA.m:346-372)
//   sim_rf_kernel         RF(t, e', g) = Re(ifft(conj(S(:, e', g)), n_fast))(t), the samples the
//                         output keeps (rcabf_sim_rf; SimUS_CUDARCA.m:374-389)
// The fields are evaluated where they are summed: no field array is stored.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "../../include/rcabf.h"

namespace rcabf {

namespace {

struct cpx {
    float x, y;
};
__device__ __forceinline__ cpx cmul(cpx a, cpx b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
__device__ __forceinline__ cpx cadd(cpx a, cpx b) { return {a.x + b.x, a.y + b.y}; }
__device__ __forceinline__ cpx cdiv(cpx a, cpx b)
{
    // scaled by the larger component of b (no overflow for the magnitudes here)
    const float s = fmaxf(fabsf(b.x), fabsf(b.y));
    const float bx = b.x / s, by = b.y / s;
    const float d = bx * bx + by * by;
    return {(a.x * bx + a.y * by) / (s * d), (a.y * bx - a.x * by) / (s * d)};
}
__device__ __forceinline__ cpx cexp(cpx a)
{
    float sn, cs;
    sincosf(a.y, &sn, &cs);
    const float m = expf(a.x);
    return {m * cs, m * sn};
}
// principal square root from the half-angle identities
//   sqrt(z) = sqrt((|z| + x) / 2) + i sign(y) sqrt((|z| - x) / 2),
// the larger of the two parts taken from its square root and the other as
// y / (2 * larger), so that neither is formed by cancellation (the ordering
// of Numerical Recipes, 2nd ed., section 5.4, "complex square root")
__device__ __forceinline__ cpx csqrt(cpx a)
{
    const float m = hypotf(a.x, a.y);
    if (!(m > 0.0f)) return {0.0f, 0.0f};
    if (a.x >= 0.0f) {
        const float u = sqrtf(0.5f * (m + a.x));
        return {u, a.y / (2.0f * u)};
    }
    const float v = copysignf(sqrtf(0.5f * (m - a.x)), a.y);
    return {a.y / (2.0f * v), v};
}
// sin(z) / z on the main lobe (|z| < pi), 0 beyond, 1 at 0
__device__ __forceinline__ cpx csinc(cpx z)
{
    const float az = hypotf(z.x, z.y);
    if (!(az > 0.0f)) return {1.0f, 0.0f};
    if (az >= 3.14159265359f) return {0.0f, 0.0f};
    float sn, cs;
    sincosf(z.x, &sn, &cs);
    const cpx s = {sn * coshf(z.y), cs * sinhf(z.y)};   // sin(x + iy)
    return cdiv(s, z);
}

// 4-term multi-Gaussian expansion of a focused element's elevation aperture
// (coefficients of the published 4-Gaussian beam model, as the reference
// simulator tabulates them, SimUS_CUDARCA.cu:10-13)
__constant__ float GA_R[4] = {0.187f, 0.288f, 0.187f, 0.288f};
__constant__ float GA_I[4] = {0.275f, -1.954f, -0.275f, 1.954f};
__constant__ float GB_R[4] = {4.558f, 8.598f, 4.558f, 8.598f};
__constant__ float GB_I[4] = {-25.59f, -7.924f, 25.59f, 7.924f};

__device__ cpx dir_flat(float theta, cpx k, float width, bool baffle)
{
    const float half = 0.5f * sinf(theta) * width;
    cpx d = csinc({half * k.x, half * k.y});
    if (baffle) {
        const float c = cosf(theta);
        d = {d.x * c, d.y * c};
    }
    return d;
}

__device__ cpx dir_focused(float r, float y, cpx k, float height, float rfocus)
{
    const cpx ik = {-k.y, k.x};                                 // i k
    const float rdn = 0.5f * (r - rfocus) / (r * rfocus);
    const cpx alpha = {ik.x * rdn, ik.y * rdn};
    const float yr = y / r, y2r = y * y / (2.0f * r);
    const cpx beta = {-ik.x * yr, -ik.y * yr};                  // -i k y / r
    const cpx gam = {ik.x * y2r, ik.y * y2r};                   // i k y^2 / (2 r)
    const cpx b2 = cmul(beta, beta);
    const float h2 = height * height;
    const float ih2 = 1.0f / h2;
    cpx sum = {0.0f, 0.0f};
#pragma unroll
    for (int g = 0; g < 4; ++g) {
        const cpx ag = {fmaf(GB_R[g], ih2, alpha.x), fmaf(GB_I[g], ih2, alpha.y)};
        // 1 / ag = conj(ag) / |ag|^2, shared by pi / ag and b^2 / (4 ag)
        const float inv = 1.0f / fmaf(ag.x, ag.x, ag.y * ag.y);
        const cpx rag = {ag.x * inv, -ag.y * inv};
        const cpx q = cmul(b2, rag);
        const cpx e = cexp({fmaf(0.25f, q.x, gam.x), fmaf(0.25f, q.y, gam.y)});
        const cpx sq = csqrt({3.14159265359f * rag.x, 3.14159265359f * rag.y});
        sum = cadd(sum, cmul({GA_R[g], GA_I[g]}, cmul(sq, e)));
    }
    return sum;
}

// The element's properties shared by all its sub-elements
struct ElemProps {
    float width, height, rfocus, lens;
    bool baffle;
};

// E(f, s, e): the field element e (sub-elements of r_ele [n_sub][5][n_ele],
// (x, y, z, az, el)) radiates to the scatterer at (xs, ys, zs) at wave number
// k (angular frequency w = Re(k) c)
__device__ cpx element_field(float xs, float ys, float zs, cpx k, float w, const float *__restrict__ r_ele, int e,
                             int n_ele, int n_sub, const ElemProps &P)
{
    float sl, cl;   // the lens delay's phase, the same for every sub-element
    sincosf(w * P.lens, &sl, &cl);
    cpx acc = {0.0f, 0.0f};
    for (int q = 0; q < n_sub; ++q) {
        const float *pe = r_ele + (int64_t)q * 5 * n_ele;
        const float xe = __ldg(&pe[e]), ye = __ldg(&pe[n_ele + e]), ze = __ldg(&pe[2 * n_ele + e]);
        const float aze = __ldg(&pe[3 * n_ele + e]), ele = __ldg(&pe[4 * n_ele + e]);
        const float dx = xs - xe, dy = ys - ye, dz = zs - ze;
        const float r = norm3df(dx, dy, dz);
        const float az = asinf(dx / r) - aze;
        const float el = asinf(dy / r) - ele;
        // Green's function exp(i k r) / r
        cpx t = cexp({-k.y * r, k.x * r});
        t = {t.x / r, t.y / r};
        t = cmul(t, dir_flat(az, k, P.width, P.baffle));
        t = cmul(t, P.rfocus > 10.0f ? dir_flat(el, k, P.width, P.baffle)
                                     : dir_focused(r, r * sinf(el), k, P.height, P.rfocus));
        acc = cadd(acc, t);
    }
    acc = cmul(acc, {cl, sl});
    // a scatterer on an element (r = 0) contributes nothing (the reference
    // zeroes the NaN it produces, SimUS_CUDARCA.m: TX(isnan(TX)) = 0)
    if (!(acc.x == acc.x) || !(acc.y == acc.y)) acc = {0.0f, 0.0f};
    return acc;
}

// out[f][s][e]; r_scat [3][n_scat] (x, y, z); r_ele [n_sub][5][n_ele] (x, y, z, az, el)
__global__ void __launch_bounds__(256) element_field_kernel(float2 *__restrict__ out,
                                                            const float *__restrict__ r_scat,
                                                            const float *__restrict__ r_ele,
                                                            const float2 *__restrict__ kwave, ElemProps P,
                                                            float c, int n_scat, int n_ele, int n_f, int n_sub)
{
    const int64_t n = (int64_t)n_f * n_scat * n_ele;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int e = (int)(i % n_ele);
        const int s = (int)((i / n_ele) % n_scat);
        const int f = (int)(i / ((int64_t)n_ele * n_scat));
        const float xs = __ldg(&r_scat[s]), ys = __ldg(&r_scat[n_scat + s]), zs = __ldg(&r_scat[2 * n_scat + s]);
        const float2 kk = __ldg(&kwave[f]);
        const cpx k = {kk.x, kk.y};
        const cpx acc = element_field(xs, ys, zs, k, k.x * c, r_ele, e, n_ele, n_sub, P);
        out[i] = make_float2(acc.x, acc.y);
    }
}

constexpr int SIM_GMAX = 16;        // transmits of a group one launch accumulates (registers)
constexpr int SIM_TX_SCAT = 32, SIM_TX_PARTS = 4;  // scatterers x element parts per block
constexpr int SIM_RX_ELE = 16, SIM_RX_PARTS = 8;   // receive elements x scatterer parts per block
constexpr int SIM_RF_THREADS = 256;

// TX[f][s][g] = T(f) b[g][s] sum_e E(f, s, e) apod[g][e] exp(i w delay[g][e]):
// one block per (frequency, 32 scatterers); its 4 warps take a quarter of
// the elements each and their sums meet in shared memory; the transmit
// weights of the block's frequency are formed once in shared memory.
__global__ void __launch_bounds__(SIM_TX_SCAT *SIM_TX_PARTS) sim_tx_kernel(
    float2 *__restrict__ tx_out, const float *__restrict__ r_scat, const float *__restrict__ bsc,
    const float *__restrict__ r_ele, const float2 *__restrict__ kwave, const float2 *__restrict__ tfac,
    const float *__restrict__ delay, const float *__restrict__ apod, ElemProps P, float c, int n_scat, int n_ele,
    int n_sub, int n_g)
{
    extern __shared__ float2 wsm[];   // [n_ele][n_g]
    __shared__ float2 part[SIM_TX_PARTS - 1][SIM_TX_SCAT][SIM_GMAX];
    const int f = blockIdx.y;
    const float2 kk = __ldg(&kwave[f]);
    const cpx k = {kk.x, kk.y};
    const float w = k.x * c;
    for (int i = threadIdx.x; i < n_ele * n_g; i += blockDim.x) {
        const int e = i / n_g, g = i % n_g;
        float sn, cs;
        sincosf(w * __ldg(&delay[(int64_t)g * n_ele + e]), &sn, &cs);
        const float a = __ldg(&apod[(int64_t)g * n_ele + e]);
        wsm[i] = make_float2(a * cs, a * sn);
    }
    __syncthreads();
    const int ls = threadIdx.x % SIM_TX_SCAT, pt = threadIdx.x / SIM_TX_SCAT;
    const int s = blockIdx.x * SIM_TX_SCAT + ls;
    cpx acc[SIM_GMAX];
#pragma unroll
    for (int g = 0; g < SIM_GMAX; ++g) acc[g] = {0.0f, 0.0f};
    if (s < n_scat) {
        const float xs = __ldg(&r_scat[s]), ys = __ldg(&r_scat[n_scat + s]), zs = __ldg(&r_scat[2 * n_scat + s]);
        for (int e = pt; e < n_ele; e += SIM_TX_PARTS) {
            const cpx E = element_field(xs, ys, zs, k, w, r_ele, e, n_ele, n_sub, P);
#pragma unroll
            for (int g = 0; g < SIM_GMAX; ++g)
                if (g < n_g) {
                    const float2 wt = wsm[e * n_g + g];
                    acc[g] = cadd(acc[g], cmul(E, {wt.x, wt.y}));
                }
        }
    }
    if (pt > 0) {
#pragma unroll
        for (int g = 0; g < SIM_GMAX; ++g) part[pt - 1][ls][g] = make_float2(acc[g].x, acc[g].y);
    }
    __syncthreads();
    if (pt == 0 && s < n_scat) {
        const float2 t2 = __ldg(&tfac[f]);
#pragma unroll
        for (int g = 0; g < SIM_GMAX; ++g)
            if (g < n_g) {
                cpx v = acc[g];
                for (int q = 0; q < SIM_TX_PARTS - 1; ++q) v = cadd(v, {part[q][ls][g].x, part[q][ls][g].y});
                const float b = __ldg(&bsc[(int64_t)g * n_scat + s]);
                v = cmul(v, {t2.x * b, t2.y * b});
                tx_out[((int64_t)f * n_scat + s) * n_g + g] = make_float2(v.x, v.y);
            }
    }
}

// S[f][e][g] = R(f) apod[g][e] sum_s E(f, s, e) TX[f][s][g]: one block per
// (frequency, 16 receive elements); its 8 thread rows take an eighth of the
// scatterers each and their sums meet in shared memory.
__global__ void __launch_bounds__(SIM_RX_ELE *SIM_RX_PARTS) sim_rx_kernel(
    float2 *__restrict__ spec, const float2 *__restrict__ tx, const float *__restrict__ r_scat,
    const float *__restrict__ r_ele, const float2 *__restrict__ kwave, const float2 *__restrict__ rfac,
    const float *__restrict__ apod, ElemProps P, float c, int n_scat, int n_ele, int n_sub, int n_g)
{
    __shared__ float2 part[SIM_RX_PARTS - 1][SIM_RX_ELE][SIM_GMAX];
    const int f = blockIdx.y;
    const int le = threadIdx.x % SIM_RX_ELE, pt = threadIdx.x / SIM_RX_ELE;
    const int e = blockIdx.x * SIM_RX_ELE + le;
    const float2 kk = __ldg(&kwave[f]);
    const cpx k = {kk.x, kk.y};
    const float w = k.x * c;
    cpx acc[SIM_GMAX];
#pragma unroll
    for (int g = 0; g < SIM_GMAX; ++g) acc[g] = {0.0f, 0.0f};
    if (e < n_ele) {
        for (int s = pt; s < n_scat; s += SIM_RX_PARTS) {
            const float xs = __ldg(&r_scat[s]), ys = __ldg(&r_scat[n_scat + s]), zs = __ldg(&r_scat[2 * n_scat + s]);
            const cpx E = element_field(xs, ys, zs, k, w, r_ele, e, n_ele, n_sub, P);
            const float2 *tp = tx + ((int64_t)f * n_scat + s) * n_g;
#pragma unroll
            for (int g = 0; g < SIM_GMAX; ++g)
                if (g < n_g) {
                    const float2 t = __ldg(&tp[g]);
                    acc[g] = cadd(acc[g], cmul(E, {t.x, t.y}));
                }
        }
    }
    if (pt > 0) {
#pragma unroll
        for (int g = 0; g < SIM_GMAX; ++g) part[pt - 1][le][g] = make_float2(acc[g].x, acc[g].y);
    }
    __syncthreads();
    if (pt == 0 && e < n_ele) {
        const float2 r2 = __ldg(&rfac[f]);
#pragma unroll
        for (int g = 0; g < SIM_GMAX; ++g)
            if (g < n_g) {
                cpx v = acc[g];
                for (int q = 0; q < SIM_RX_PARTS - 1; ++q) v = cadd(v, {part[q][le][g].x, part[q][le][g].y});
                const float a = __ldg(&apod[(int64_t)g * n_ele + e]);
                v = cmul(v, {r2.x * a, r2.y * a});
                spec[((int64_t)f * n_ele + e) * n_g + g] = make_float2(v.x, v.y);
            }
    }
}

// out[g][e][i]: the sample t(i) of Re(ifft(conj(S[:, e, g]), n_fast)), i.e.
// (1/n_fast) sum_f (Re S_f cos(2 pi f t / n_fast) + Im S_f sin(2 pi f t / n_fast))
// with the twiddle table tw[m] = exp(2 pi i m / n_fast).  sub = 0: t = i for
// i < n_out (the RF, zero from n_fast on); sub > 0: t = sub (i / 2) + i % 2
// (the quadrature-sampled interleave of RF(1:sub:end) and RF(2:sub:end)).
// One block per (receive element, transmit) and 256 output samples; the
// column's spectrum and, when it fits (TW_SMEM), the twiddle table are
// staged in shared memory (the samples of a warp read scattered twiddles).
template <bool TW_SMEM>
__global__ void __launch_bounds__(SIM_RF_THREADS) sim_rf_kernel(float *__restrict__ out,
                                                                const float2 *__restrict__ spec,
                                                                const float2 *__restrict__ tw, int n_f, int n_ele,
                                                                int n_g, int n_fast, int sub, int n_out)
{
    extern __shared__ float2 col[];   // [n_f], then [n_fast] twiddles
    const int eg = blockIdx.y;        // e * n_g + g
    const int e = eg / n_g, g = eg % n_g;
    for (int f = threadIdx.x; f < n_f; f += blockDim.x) col[f] = spec[(int64_t)f * n_ele * n_g + eg];
    float2 *tws = col + n_f;
    if constexpr (TW_SMEM)
        for (int m = threadIdx.x; m < n_fast; m += blockDim.x) tws[m] = __ldg(&tw[m]);
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_out) return;
    const int t = sub == 0 ? i : sub * (i / 2) + (i % 2);
    float acc = 0.0f;
    if (t < n_fast) {
        int m = 0;   // f t mod n_fast
        for (int f = 0; f < n_f; ++f) {
            const float2 x = col[f];
            const float2 r = TW_SMEM ? tws[m] : __ldg(&tw[m]);
            acc = fmaf(x.x, r.x, fmaf(x.y, r.y, acc));
            m += t;
            if (m >= n_fast) m -= n_fast;
        }
        acc *= 1.0f / (float)n_fast;
    }
    out[((int64_t)g * n_ele + e) * n_out + i] = acc;
}

}  // namespace

}  // namespace rcabf

extern "C" int rcabf_sim_element_field(void *out, const float *r_scat, const float *r_ele, const void *kwave,
                                       float width, float height, float rfocus, int baffle, float lens,
                                       float speed_of_sound, int64_t n_scat, int64_t n_ele, int64_t n_f,
                                       int64_t n_sub, void *stream)
{
    if (!out || !r_scat || !r_ele || !kwave) return RCABF_ERR_INVALID_ARGUMENT;
    if (n_scat < 1 || n_ele < 1 || n_f < 1 || n_sub < 1 || n_scat > INT32_MAX || n_ele > INT32_MAX ||
        n_f > INT32_MAX || n_sub > 64)
        return RCABF_ERR_SHAPE_MISMATCH;
    int dev = 0, n_sm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    const int64_t n = n_f * n_scat * n_ele;
    const int64_t blocks = std::min<int64_t>((n + 255) / 256, (int64_t)n_sm * 8);
    const rcabf::ElemProps P{width, height, rfocus, lens, baffle == 1};
    rcabf::element_field_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<float2 *>(out), r_scat, r_ele, reinterpret_cast<const float2 *>(kwave), P, speed_of_sound,
        (int)n_scat, (int)n_ele, (int)n_f, (int)n_sub);
    return cudaGetLastError() == cudaSuccess ? RCABF_OK : RCABF_ERR_CUDA;
}

extern "C" int rcabf_sim_tx_field(void *tx_out, const float *r_scat, const float *bsc, const float *r_ele,
                                  const void *kwave, const void *tx_factor, const float *delay, const float *apod,
                                  int64_t n_tx, float width, float height, float rfocus, int baffle, float lens,
                                  float speed_of_sound, int64_t n_scat, int64_t n_ele, int64_t n_f, int64_t n_sub,
                                  void *stream)
{
    if (!tx_out || !r_scat || !bsc || !r_ele || !kwave || !tx_factor || !delay || !apod)
        return RCABF_ERR_INVALID_ARGUMENT;
    if (n_scat < 1 || n_ele < 1 || n_f < 1 || n_sub < 1 || n_tx < 1 || n_tx > rcabf::SIM_GMAX || n_sub > 64 ||
        n_scat > INT32_MAX || n_f > 65535 || n_ele * n_tx > 4096)
        return RCABF_ERR_SHAPE_MISMATCH;
    const rcabf::ElemProps P{width, height, rfocus, lens, baffle == 1};
    const dim3 grid((unsigned)((n_scat + rcabf::SIM_TX_SCAT - 1) / rcabf::SIM_TX_SCAT), (unsigned)n_f);
    rcabf::sim_tx_kernel<<<grid, rcabf::SIM_TX_SCAT * rcabf::SIM_TX_PARTS, (size_t)(n_ele * n_tx * 8),
                           (cudaStream_t)stream>>>(
        reinterpret_cast<float2 *>(tx_out), r_scat, bsc, r_ele, reinterpret_cast<const float2 *>(kwave),
        reinterpret_cast<const float2 *>(tx_factor), delay, apod, P, speed_of_sound, (int)n_scat, (int)n_ele,
        (int)n_sub, (int)n_tx);
    return cudaGetLastError() == cudaSuccess ? RCABF_OK : RCABF_ERR_CUDA;
}

extern "C" int rcabf_sim_rx_spectrum(void *spec_out, const void *tx_field, const float *r_scat, const float *r_ele,
                                     const void *kwave, const void *rx_factor, const float *apod, int64_t n_tx,
                                     float width, float height, float rfocus, int baffle, float lens,
                                     float speed_of_sound, int64_t n_scat, int64_t n_ele, int64_t n_f, int64_t n_sub,
                                     void *stream)
{
    if (!spec_out || !tx_field || !r_scat || !r_ele || !kwave || !rx_factor || !apod)
        return RCABF_ERR_INVALID_ARGUMENT;
    if (n_scat < 1 || n_ele < 1 || n_f < 1 || n_sub < 1 || n_tx < 1 || n_tx > rcabf::SIM_GMAX || n_sub > 64 ||
        n_scat > INT32_MAX || n_ele > INT32_MAX || n_f > 65535)
        return RCABF_ERR_SHAPE_MISMATCH;
    const rcabf::ElemProps P{width, height, rfocus, lens, baffle == 1};
    const dim3 grid((unsigned)((n_ele + rcabf::SIM_RX_ELE - 1) / rcabf::SIM_RX_ELE), (unsigned)n_f);
    rcabf::sim_rx_kernel<<<grid, rcabf::SIM_RX_ELE * rcabf::SIM_RX_PARTS, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<float2 *>(spec_out), reinterpret_cast<const float2 *>(tx_field), r_scat, r_ele,
        reinterpret_cast<const float2 *>(kwave), reinterpret_cast<const float2 *>(rx_factor), apod, P,
        speed_of_sound, (int)n_scat, (int)n_ele, (int)n_sub, (int)n_tx);
    return cudaGetLastError() == cudaSuccess ? RCABF_OK : RCABF_ERR_CUDA;
}

extern "C" int rcabf_sim_rf(float *out, const void *spec, const void *twiddle, int64_t n_f, int64_t n_ele,
                            int64_t n_tx, int64_t n_fast, int32_t sub, int64_t n_out, void *stream)
{
    if (!out || !spec || !twiddle) return RCABF_ERR_INVALID_ARGUMENT;
    if (n_f < 1 || n_ele < 1 || n_tx < 1 || n_fast < 1 || n_out < 1 || sub < 0 || n_f > n_fast ||
        n_f * 8 > 48 * 1024 || n_ele * n_tx > 65535 || n_fast > INT32_MAX / 2 || n_out > INT32_MAX)
        return RCABF_ERR_SHAPE_MISMATCH;
    const dim3 grid((unsigned)((n_out + rcabf::SIM_RF_THREADS - 1) / rcabf::SIM_RF_THREADS), (unsigned)(n_ele * n_tx));
    const size_t smem_tw = (size_t)(n_f + n_fast) * 8;
    const auto *sp = reinterpret_cast<const float2 *>(spec);
    const auto *tw = reinterpret_cast<const float2 *>(twiddle);
    if (smem_tw <= 96 * 1024) {
        auto k = rcabf::sim_rf_kernel<true>;
        if (smem_tw > 48 * 1024 &&
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_tw) != cudaSuccess)
            return RCABF_ERR_CUDA;
        k<<<grid, rcabf::SIM_RF_THREADS, smem_tw, (cudaStream_t)stream>>>(out, sp, tw, (int)n_f, (int)n_ele,
                                                                          (int)n_tx, (int)n_fast, sub, (int)n_out);
    } else {
        rcabf::sim_rf_kernel<false><<<grid, rcabf::SIM_RF_THREADS, (size_t)(n_f * 8), (cudaStream_t)stream>>>(
            out, sp, tw, (int)n_f, (int)n_ele, (int)n_tx, (int)n_fast, sub, (int)n_out);
    }
    return cudaGetLastError() == cudaSuccess ? RCABF_OK : RCABF_ERR_CUDA;
}
