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
// per element and the transmit delays / apodisations are applied afterwards
// as one batched complex GEMM per frequency (the transmit field is linear in
// them), which removes the transmit count from the transcendental work.
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
// principal square root: sqrt(|z|) e^{i arg(z) / 2}
__device__ __forceinline__ cpx csqrt(cpx a)
{
    const float m = sqrtf(hypotf(a.x, a.y));
    float sn, cs;
    sincosf(0.5f * atan2f(a.y, a.x), &sn, &cs);
    return {m * cs, m * sn};
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
    cpx sum = {0.0f, 0.0f};
#pragma unroll
    for (int g = 0; g < 4; ++g) {
        const cpx ag = {GB_R[g] / h2 + alpha.x, GB_I[g] / h2 + alpha.y};
        const cpx e = cexp(cadd(cdiv(b2, {4.0f * ag.x, 4.0f * ag.y}), gam));
        const cpx sq = csqrt(cdiv({3.14159265359f, 0.0f}, ag));
        sum = cadd(sum, cmul({GA_R[g], GA_I[g]}, cmul(sq, e)));
    }
    return sum;
}

// out[f][s][e]; r_scat [3][n_scat] (x, y, z); r_ele [n_sub][5][n_ele] (x, y, z, az, el)
__global__ void __launch_bounds__(256) element_field_kernel(float2 *__restrict__ out,
                                                            const float *__restrict__ r_scat,
                                                            const float *__restrict__ r_ele,
                                                            const float2 *__restrict__ kwave, float width,
                                                            float height, float rfocus, int baffle, float lens,
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
        const float w = k.x * c;
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
            t = cmul(t, dir_flat(az, k, width, baffle == 1));
            t = cmul(t, rfocus > 10.0f ? dir_flat(el, k, width, baffle == 1)
                                       : dir_focused(r, r * sinf(el), k, height, rfocus));
            float sl, cl;
            sincosf(w * lens, &sl, &cl);
            t = cmul(t, {cl, sl});
            acc = cadd(acc, t);
        }
        // a scatterer on an element (r = 0) contributes nothing (the reference
        // zeroes the NaN it produces, SimUS_CUDARCA.m: TX(isnan(TX)) = 0)
        if (!(acc.x == acc.x) || !(acc.y == acc.y)) acc = {0.0f, 0.0f};
        out[i] = make_float2(acc.x, acc.y);
    }
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
    rcabf::element_field_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(
        reinterpret_cast<float2 *>(out), r_scat, r_ele, reinterpret_cast<const float2 *>(kwave), width, height,
        rfocus, baffle, lens, speed_of_sound, (int)n_scat, (int)n_ele, (int)n_f, (int)n_sub);
    return cudaGetLastError() == cudaSuccess ? RCABF_OK : RCABF_ERR_CUDA;
}
