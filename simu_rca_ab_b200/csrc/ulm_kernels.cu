// Ultrasound localisation microscopy (ULM) super-localisation on the GPU,
// the downstream consumer of the clutter-filtered beamformed ensemble
// (Python/superloc/superloc.py).  Maps are stacks of 2-D frames stored with
// z fastest, then x, then frame: element (z, x, t) at z + nz * (x + nx * t),
// the column-major order the reference's ArrayFire arrays use, so linear
// indices mean the same thing on both sides.
//
//   rcabf_ulm_psf_corr   PsfCorrMap2D (superloc.py:12-48): PSF correlation
//                        map normalised by the local energy and the PSF norm
//   rcabf_ulm_ensemble   sqrt|Hann-smoothed lag-1 product| along frames
//                        (superloc.py:114-120)
//   rcabf_ulm_regional_max  ImRegionalMax (superloc.py:51-53)
//   rcabf_ulm_detect     regional maxima of the maps inside the border ROI
//                        (superloc.py:51-53, 122-136), compacted
//   rcabf_ulm_gauss_fit  Hann-weighted log-parabola fit of every detection
//                        (superloc.py:56-100, 170-213)
//   rcabf_ulm_density    density / velocity histograms (superloc.py:216-402)
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "../../include/rcabf.h"

namespace rcabf {
namespace {

constexpr int ULM_MAX_PSF = 33;                      // largest PSF extent per axis
constexpr int CORR_TZ = 32, CORR_TX = 8;             // output tile (z x x) of one CTA

// out(z, x) = sum_{a, b} iq(z + kz/2 - a, x + kx/2 - b) conj(psf(a, b)),
// energy(z, x) = sum over the same footprint of |iq|^2 (zero outside the
// frame): ArrayFire's same-size convolution.  One CTA per 32 x 8 output tile
// of one frame; the input tile with its halo and the PSF sit in shared memory.
__global__ void __launch_bounds__(CORR_TZ * CORR_TX) psf_corr_kernel(float2 *__restrict__ out,
                                                                     const float2 *__restrict__ iq,
                                                                     const float2 *__restrict__ psf, float inv_psf_norm,
                                                                     int nz, int nx, int kz, int kx)
{
    extern __shared__ float2 sm[];
    const int hz = CORR_TZ + kz - 1, hx = CORR_TX + kx - 1;
    float2 *tile = sm;                  // [hx][hz]
    float2 *ker = sm + hz * hx;         // [kx][kz], conjugated
    const int t = blockIdx.z;
    const int z0 = blockIdx.x * CORR_TZ, x0 = blockIdx.y * CORR_TX;
    const int tid = threadIdx.y * CORR_TZ + threadIdx.x;
    const float2 *frame = iq + (int64_t)t * nz * nx;
    // tile row r holds input z = z0 + kz/2 - (kz - 1) + r; column c holds
    // x = x0 + kx/2 - (kx - 1) + c
    const int zb = z0 + kz / 2 - (kz - 1), xb = x0 + kx / 2 - (kx - 1);
    for (int i = tid; i < hz * hx; i += CORR_TZ * CORR_TX) {
        const int r = i % hz, c = i / hz;
        const int z = zb + r, x = xb + c;
        tile[i] = (z >= 0 && z < nz && x >= 0 && x < nx) ? frame[(int64_t)x * nz + z] : make_float2(0.f, 0.f);
    }
    for (int i = tid; i < kz * kx; i += CORR_TZ * CORR_TX) {
        const float2 p = psf[i];   // psf(a, b) at a + kz * b
        ker[i] = make_float2(p.x, -p.y);
    }
    __syncthreads();
    const int z = z0 + threadIdx.x, x = x0 + threadIdx.y;
    if (z >= nz || x >= nx) return;
    float re = 0.f, im = 0.f, en = 0.f;
    for (int b = 0; b < kx; ++b) {
        // input column x + kx/2 - b  ->  tile column threadIdx.y + kx - 1 - b
        const float2 *col = tile + (threadIdx.y + kx - 1 - b) * hz + threadIdx.x + kz - 1;
        const float2 *kc = ker + b * kz;
        for (int a = 0; a < kz; ++a) {
            const float2 v = col[-a];
            const float2 k = kc[a];
            re = fmaf(v.x, k.x, fmaf(-v.y, k.y, re));
            im = fmaf(v.x, k.y, fmaf(v.y, k.x, im));
            en = fmaf(v.x, v.x, fmaf(v.y, v.y, en));
        }
    }
    // (num / sqrt(energy)) / |psf|, IEEE division as the reference's
    const float s = sqrtf(en);
    out[((int64_t)t * nx + x) * nz + z] = make_float2(re / s * inv_psf_norm, im / s * inv_psf_norm);
}

// out(z, x, t) = sqrt|sum_f ker(f) p(t + K/2 - f)|, p(u) = m(u) conj(m(u + 1))
// for 0 <= u < nt - 1 (zero outside); t < nt - 1.
__global__ void ensemble_kernel(float *__restrict__ out, const float2 *__restrict__ m,
                                const float *__restrict__ ker, int nker, int64_t plane, int nt)
{
    const int64_t n = plane * (nt - 1);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = i % plane;
        const int t = (int)(i / plane);
        float re = 0.f, im = 0.f;
        for (int f = 0; f < nker; ++f) {
            const int u = t + nker / 2 - f;
            if (u < 0 || u >= nt - 1) continue;
            const float2 a = m[(int64_t)u * plane + p], b = m[(int64_t)(u + 1) * plane + p];
            const float pr = fmaf(a.x, b.x, a.y * b.y), pi = fmaf(a.y, b.x, -a.x * b.y);   // a conj(b)
            re = fmaf(ker[f], pr, re);
            im = fmaf(ker[f], pi, im);
        }
        out[i] = sqrtf(hypotf(re, im));
    }
}

// value of map m at (z, x) of frame plane `t0`, -inf outside the frame
__device__ __forceinline__ float at_or_lowest(const float *m, int z, int x, int nz, int nx)
{
    return (z >= 0 && z < nz && x >= 0 && x < nx) ? m[(int64_t)x * nz + z] : -INFINITY;
}
// dilate(m, ones(3, 3)) == m at (z, x)
__device__ __forceinline__ bool is_regional_max(const float *m, int z, int x, int nz, int nx)
{
    const float c = m[(int64_t)x * nz + z];
    float d = -INFINITY;
#pragma unroll
    for (int b = -1; b <= 1; ++b)
#pragma unroll
        for (int a = -1; a <= 1; ++a) d = fmaxf(d, at_or_lowest(m, z + a, x + b, nz, nx));
    return d == c;   // false for NaN, as the reference's comparison
}

// bw(z, x, t) = dilate(m, ones(3, 3)) == m
__global__ void regmax_kernel(uint8_t *__restrict__ bw, const float *__restrict__ m, int nz, int nx, int64_t n)
{
    const int64_t plane = (int64_t)nz * nx;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int z = (int)(i % nz), x = (int)((i / nz) % nx);
        bw[i] = is_regional_max(m + (i / plane) * plane, z, x, nz, nx) ? 1 : 0;
    }
}

// Candidates: fit 0: regmax(C) and a regional maximum of E within 3 x 3;
// fit 1: regmax(E); both inside the ROI [edge, n - edge) of z and x.
// Appends (linear index, |value of the fitted map|) in any order.
__global__ void detect_kernel(int64_t *__restrict__ lin, float *__restrict__ val, unsigned long long *__restrict__ count,
                              const float *__restrict__ C, const float *__restrict__ E, int nz, int nx, int nt1,
                              int edge, int fit, int64_t capacity)
{
    const int64_t plane = (int64_t)nz * nx, n = plane * nt1;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int z = (int)(i % nz), x = (int)((i / nz) % nx);
        const int64_t t = i / plane;
        if (z < edge || z >= nz - edge || x < edge || x >= nx - edge) continue;
        const float *c = C + t * plane, *e = E + t * plane;
        bool hit;
        if (fit == 0) {
            hit = is_regional_max(c, z, x, nz, nx);
            if (hit) {
                bool any = false;
                for (int b = -1; b <= 1 && !any; ++b)
                    for (int a = -1; a <= 1 && !any; ++a) {
                        const int zz = z + a, xx = x + b;
                        if (zz >= 0 && zz < nz && xx >= 0 && xx < nx) any = is_regional_max(e, zz, xx, nz, nx);
                    }
                hit = any;
            }
        } else {
            hit = is_regional_max(e, z, x, nz, nx);
        }
        if (!hit) continue;
        const unsigned long long k = atomicAdd(count, 1ull);
        if ((int64_t)k < capacity) {
            lin[k] = i;
            val[k] = fabsf((fit == 0 ? c : e)[(int64_t)x * nz + z]);
        }
    }
}

// One thread per detection (in the caller's order).  The reference reads
// the detection's coordinates from meshgrid(ix, iz, it) flattened in Fortran
// order at the mask's column-major index (superloc.py:140-168):
//   ix = (L mod n0 n1) div n1, iz = L mod n1, it = L div n0 n1
// (n0, n1 = the map's first two extents), i.e. (x, z) for square maps.
// consts: hann[(2e+1)^2] at izr + (2e+1) ixr, roi[2e+1], ata_x_inv[9],
// ata_z_inv[9] (row-major).
__global__ void gauss_fit_kernel(float *__restrict__ pos, const int64_t *__restrict__ lin,
                                 const float *__restrict__ val, int64_t n, const float *__restrict__ map, int nz, int nx,
                                 int64_t n_map, int edge, const float *__restrict__ consts)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int w = 2 * edge + 1;
    const float *hann = consts, *roi = consts + w * w, *axi = roi + w, *azi = axi + 9;
    const int64_t L = lin[i], n01 = (int64_t)nz * nx;
    const int64_t ix = (L % n01) / nx, iz = L % nx, it = L / n01;
    float ax0 = 0.f, ax1 = 0.f, ax2 = 0.f, az0 = 0.f, az1 = 0.f, az2 = 0.f;
    for (int ixr = 0; ixr < w; ++ixr) {
        for (int izr = 0; izr < w; ++izr) {
            const int64_t idx = (iz - edge + izr) + (ix - edge + ixr) * nz + it * n01;
            // a neighbour outside the map (possible only for non-square maps,
            // where the reference's index mapping scrambles x and z) reads NaN
            const float lg = (idx >= 0 && idx < n_map) ? logf(fabsf(map[idx])) : NAN;
            const float h = hann[izr + w * ixr];
            const float rx = roi[ixr], rz = roi[izr];
            const float lh = lg * h;
            ax0 += lh;
            ax1 += lh * rx;
            ax2 += lh * rx * rx;
            az0 += lh;
            az1 += lh * rz;
            az2 += lh * rz * rz;
        }
    }
    const float mx1 = axi[3] * ax0 + axi[4] * ax1 + axi[5] * ax2;
    const float mx2 = axi[6] * ax0 + axi[7] * ax1 + axi[8] * ax2;
    const float mz1 = azi[3] * az0 + azi[4] * az1 + azi[5] * az2;
    const float mz2 = azi[6] * az0 + azi[7] * az1 + azi[8] * az2;
    pos[i] = (float)ix + (-0.5f * mx1 / mx2);
    pos[n + i] = 0.0f;
    pos[2 * n + i] = (float)iz + (-0.5f * mz1 / mz2);
    pos[3 * n + i] = val[i];
    pos[4 * n + i] = (float)it;
}

// numpy's float64 -> int16 cast on x86-64: truncation to int32 (an
// out-of-range or NaN value gives INT32_MIN), then the low 16 bits
__device__ __forceinline__ int bin_index(double v, double lo, double step, int64_t nbin)
{
    const double q = (v - lo) / step;
    int32_t i32;
    if (!(q > -2147483649.0 && q < 2147483648.0)) i32 = INT32_MIN;
    else i32 = (int32_t)trunc(q);
    int i = (int16_t)(uint16_t)((uint32_t)i32 & 0xffffu);
    i = i > 0 ? i : 0;                                         // (i > 0) * i
    const int64_t d = nbin - i;                                // ((n - i) > 0) * i + ((n - i) < 0) * (n - 1)
    return (int)((d > 0 ? i : 0) + (d < 0 ? nbin - 1 : 0));
}

// dens[z][x][y][t] += 1 (vel[c][z][x][y][t] += v_c) per position; pos rows
// 0, 1, 2 (and 4 when binning time) are x, y, z (and t)
__global__ void density_kernel(double *__restrict__ dens, double *__restrict__ vel, const double *__restrict__ pos,
                               int64_t n, const double *__restrict__ vin, rcabf_ulm_bins b, int use_t)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double *p = pos + i * b.pos_rows;
    const int ix = bin_index(p[0], b.min[0], b.step[0], b.n[0]);
    const int iy = bin_index(p[1], b.min[1], b.step[1], b.n[1]);
    const int iz = bin_index(p[2], b.min[2], b.step[2], b.n[2]);
    const int itb = use_t ? bin_index(p[4], b.min[3], b.step[3], b.n[3]) : 0;
    const int64_t nt = use_t ? b.n[3] : 1;
    const int64_t cell = (((int64_t)iz * b.n[0] + ix) * b.n[1] + iy) * nt + itb;
    atomicAdd(dens + cell, 1.0);
    if (vel) {
        const int64_t ncell = b.n[2] * b.n[0] * b.n[1] * nt;
        for (int c = 0; c < 3; ++c) atomicAdd(vel + c * ncell + cell, vin[i * b.vel_rows + c]);
    }
}

int grid_for(int64_t n, int threads)
{
    int dev = 0, n_sm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    const int64_t g = (n + threads - 1) / threads;
    return (int)(g < (int64_t)n_sm * 16 ? (g > 0 ? g : 1) : (int64_t)n_sm * 16);
}

int status_of(cudaError_t e) { return e == cudaSuccess ? RCABF_OK : RCABF_ERR_CUDA; }

}  // namespace
}  // namespace rcabf

using namespace rcabf;

extern "C" int rcabf_ulm_psf_corr(void *corr, const void *iq, const void *psf, float psf_norm, int64_t nz, int64_t nx,
                                  int64_t nt, int32_t kz, int32_t kx, void *stream)
{
    if (!corr || !iq || !psf) return RCABF_ERR_INVALID_ARGUMENT;
    if (nz < 1 || nx < 1 || nt < 1 || kz < 1 || kx < 1 || nz > INT32_MAX || nx > INT32_MAX || nt > 65535)
        return RCABF_ERR_SHAPE_MISMATCH;
    if (kz > ULM_MAX_PSF || kx > ULM_MAX_PSF) return RCABF_ERR_UNSUPPORTED;
    if (!(psf_norm > 0.0f)) return RCABF_ERR_INVALID_ARGUMENT;
    const size_t smem = ((size_t)(CORR_TZ + kz - 1) * (CORR_TX + kx - 1) + (size_t)kz * kx) * sizeof(float2);
    cudaError_t e = cudaFuncSetAttribute(psf_corr_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return RCABF_ERR_CUDA;
    const dim3 grid((unsigned)((nz + CORR_TZ - 1) / CORR_TZ), (unsigned)((nx + CORR_TX - 1) / CORR_TX), (unsigned)nt);
    psf_corr_kernel<<<grid, dim3(CORR_TZ, CORR_TX), smem, (cudaStream_t)stream>>>(
        reinterpret_cast<float2 *>(corr), reinterpret_cast<const float2 *>(iq), reinterpret_cast<const float2 *>(psf),
        1.0f / psf_norm, (int)nz, (int)nx, kz, kx);
    return status_of(cudaGetLastError());
}

extern "C" int rcabf_ulm_ensemble(float *out, const void *map, const float *ker, int32_t nker, int64_t nz, int64_t nx,
                                  int64_t nt, void *stream)
{
    if (!out || !map || !ker) return RCABF_ERR_INVALID_ARGUMENT;
    if (nz < 1 || nx < 1 || nt < 2 || nker < 1 || nt > INT32_MAX) return RCABF_ERR_SHAPE_MISMATCH;
    const int64_t plane = nz * nx, n = plane * (nt - 1);
    ensemble_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(out, reinterpret_cast<const float2 *>(map), ker,
                                                                       nker, plane, (int)nt);
    return status_of(cudaGetLastError());
}

extern "C" int rcabf_ulm_regional_max(uint8_t *bw, const float *map, int64_t nz, int64_t nx, int64_t nt, void *stream)
{
    if (!bw || !map) return RCABF_ERR_INVALID_ARGUMENT;
    if (nz < 1 || nx < 1 || nt < 1 || nz > INT32_MAX || nx > INT32_MAX) return RCABF_ERR_SHAPE_MISMATCH;
    const int64_t n = nz * nx * nt;
    regmax_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(bw, map, (int)nz, (int)nx, n);
    return status_of(cudaGetLastError());
}

extern "C" int rcabf_ulm_detect(int64_t *lin, float *val, uint64_t *count, const float *corr_ens, const float *env_ens,
                                int64_t nz, int64_t nx, int64_t nt, int32_t edge, int32_t fit, int64_t capacity,
                                void *stream)
{
    if (!lin || !val || !count || !env_ens || (fit == 0 && !corr_ens)) return RCABF_ERR_INVALID_ARGUMENT;
    if (fit != 0 && fit != 1) return RCABF_ERR_INVALID_ARGUMENT;
    if (nz < 1 || nx < 1 || nt < 1 || edge < 0 || capacity < 0 || nz > INT32_MAX || nx > INT32_MAX)
        return RCABF_ERR_SHAPE_MISMATCH;
    const int64_t n = nz * nx * nt;
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(uint64_t), (cudaStream_t)stream);
    if (e != cudaSuccess) return RCABF_ERR_CUDA;
    detect_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(
        lin, val, reinterpret_cast<unsigned long long *>(count), fit == 0 ? corr_ens : env_ens, env_ens, (int)nz,
        (int)nx, (int)nt, edge, fit, capacity);
    return status_of(cudaGetLastError());
}

extern "C" int rcabf_ulm_gauss_fit(float *pos, const int64_t *lin, const float *val, int64_t n, const float *map,
                                   int64_t nz, int64_t nx, int64_t nt, int32_t edge, const float *consts, void *stream)
{
    if (!pos || (n > 0 && (!lin || !val || !map || !consts))) return RCABF_ERR_INVALID_ARGUMENT;
    if (nz < 1 || nx < 1 || nt < 1 || edge < 0 || n < 0 || nz > INT32_MAX || nx > INT32_MAX)
        return RCABF_ERR_SHAPE_MISMATCH;
    if (n == 0) return RCABF_OK;
    gauss_fit_kernel<<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(pos, lin, val, n, map, (int)nz,
                                                                                     (int)nx, nz * nx * nt, edge, consts);
    return status_of(cudaGetLastError());
}

extern "C" int rcabf_ulm_density(double *dens, double *vel, const double *pos, int64_t n, const double *vel_in,
                                 const rcabf_ulm_bins *bins, int32_t use_t, void *stream)
{
    if (!dens || !bins || (n > 0 && !pos) || (vel && n > 0 && !vel_in)) return RCABF_ERR_INVALID_ARGUMENT;
    if (bins->struct_size != (int32_t)sizeof(rcabf_ulm_bins)) return RCABF_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < (use_t ? 4 : 3); ++k)
        if (bins->n[k] < 1 || !(bins->step[k] != 0.0)) return RCABF_ERR_SHAPE_MISMATCH;
    if (bins->pos_rows < (use_t ? 5 : 3) || (vel && bins->vel_rows < 3)) return RCABF_ERR_SHAPE_MISMATCH;
    if (n == 0) return RCABF_OK;
    density_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(dens, vel, pos, n, vel_in, *bins,
                                                                                   use_t);
    return status_of(cudaGetLastError());
}
