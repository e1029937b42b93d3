// Auxiliary kernels of librcabf: channel-data ingest, per-tile window range
// tables, the apodisation-sum mask, and an FP32 FMA throughput probe.
#include <algorithm>

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "das_kernels.cuh"
#include "launchers.h"

namespace rcabf {

// ------------------------------------------------------------------------
// Ingest: caller layout [frame][tx][ele][sample] (any rcabf_iq_dtype) ->
// slabs [tx][ele][frame block][sample][frame in block] in the storage type.
// One block moves 64 samples x FB frames of one (tx, ele) through shared
// memory so that both the reads (along samples) and the writes (along
// sample-major, frame-minor rows) are coalesced.
// ------------------------------------------------------------------------
template <int STORE> __device__ __forceinline__ typename StoreT<STORE>::T from_f2(float2 v);
template <> __device__ __forceinline__ float2 from_f2<ST_F32>(float2 v) { return v; }
template <> __device__ __forceinline__ __half2 from_f2<ST_F16>(float2 v) { return __float22half2_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat162 from_f2<ST_BF16>(float2 v) { return __float22bfloat162_rn(v); }

constexpr int INGEST_NS = 64;
constexpr int INGEST_FCHUNK = 64;    // frames of a block one CTA moves
constexpr int INGEST_MAX_FB = 256;

// grid.y = frame block x chunk of up to INGEST_FCHUNK of its frames
template <int STORE, int IQ>
__global__ void __launch_bounds__(256) ingest_kernel(const IngestParams p)
{
    using T = typename StoreT<STORE>::T;
    __shared__ float2 tile[INGEST_FCHUNK][INGEST_NS + 1];
    const int n_base = blockIdx.x * INGEST_NS;
    const int n_chunk = (p.fb + INGEST_FCHUNK - 1) / INGEST_FCHUNK;
    const int fb = blockIdx.y / n_chunk;
    const int f0 = (blockIdx.y % n_chunk) * INGEST_FCHUNK;   // first frame of the chunk within the block
    const int te = blockIdx.z;
    const int tx = te / p.n_ele, ele = te % p.n_ele;
    const int FB = p.fb;
    const int FC = min(INGEST_FCHUNK, FB - f0);              // frames of this chunk
    for (int i = threadIdx.x; i < FC * INGEST_NS; i += blockDim.x) {
        const int fi = i / INGEST_NS, nl = i % INGEST_NS;
        const int64_t f = (int64_t)fb * FB + f0 + fi;
        const int n = n_base + nl;
        float2 v = make_float2(0.f, 0.f);
        if (f < p.n_frame && n < p.n_sample)
            v = load_iq<IQ>(p.iq, ((f * p.n_tx + tx) * (int64_t)p.n_ele + ele) * p.n_sample + n);
        tile[fi][nl] = v;
    }
    __syncthreads();
    T *slab = reinterpret_cast<T *>(reinterpret_cast<char *>(p.S) +
                                    (((int64_t)tx * p.n_ele + ele) * p.n_fb + fb) * p.slab_bytes);
    const int n_rows = max(p.n_rows, p.n_sample);
    T *slab2 = p.S2 == nullptr ? nullptr
                               : reinterpret_cast<T *>(reinterpret_cast<char *>(p.S2) +
                                                       (((int64_t)tx * p.n_ele + ele) * p.n_fb + fb) * p.slab_bytes);
    for (int i = threadIdx.x; i < FC * INGEST_NS; i += blockDim.x) {
        const int nl = i / FC, fi = i % FC;
        const int n = n_base + nl;
        if (n < n_rows) {
            const float2 v = tile[fi][nl];
            slab[(int64_t)n * FB + f0 + fi] = from_f2<STORE>(v);   // zeros past the record
            if (slab2) slab2[(int64_t)n * FB + f0 + fi] = from_f2<STORE>(make_float2(-v.y, v.x));
        }
    }
}

template <int STORE>
static cudaError_t launch_ingest_store(const IngestParams &p, cudaStream_t st)
{
    const int n_chunk = (p.fb + INGEST_FCHUNK - 1) / INGEST_FCHUNK;
    dim3 grid((std::max(p.n_rows, p.n_sample) + INGEST_NS - 1) / INGEST_NS, p.n_fb * n_chunk, p.n_tx * p.n_ele);
    switch (p.iq_dtype) {
    case 0: ingest_kernel<STORE, 0><<<grid, 256, 0, st>>>(p); break;
    case 1: ingest_kernel<STORE, 1><<<grid, 256, 0, st>>>(p); break;
    case 2: ingest_kernel<STORE, 2><<<grid, 256, 0, st>>>(p); break;
    case 3: ingest_kernel<STORE, 3><<<grid, 256, 0, st>>>(p); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_ingest(const IngestParams &p, int store, cudaStream_t st)
{
    if (p.fb < 1 || p.fb > INGEST_MAX_FB || (int64_t)p.n_fb * ((p.fb + INGEST_FCHUNK - 1) / INGEST_FCHUNK) > 65535 ||
        p.n_tx * p.n_ele > 65535)
        return cudaErrorInvalidValue;
    switch (store) {
    case ST_F32: return launch_ingest_store<ST_F32>(p, st);
    case ST_F16: return launch_ingest_store<ST_F16>(p, st);
    case ST_BF16: return launch_ingest_store<ST_BF16>(p, st);
    default: return cudaErrorInvalidValue;
    }
}

// ------------------------------------------------------------------------
// Window range tables: (min, max) of the table delay over each tile's keys,
// valid entries only.  tab is [rows][n_a * n_z]; out is [rows][tiles_a][tiles_z].
// ------------------------------------------------------------------------
__global__ void range_kernel(const RangeParams p)
{
    const int64_t n_out = (int64_t)p.rows * p.tiles_a * p.tiles_z;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_out) return;
    const int tzi = (int)(i % p.tiles_z);
    const int tai = (int)((i / p.tiles_z) % p.tiles_a);
    const int64_t row = i / ((int64_t)p.tiles_z * p.tiles_a);
    float lo = __int_as_float(0x7f800000), hi = -lo;
    for (int a = 0; a < p.ta; ++a) {
        const int64_t ia = (int64_t)tai * p.ta + a;
        if (ia >= p.n_a) break;
        for (int z = 0; z < p.tz; ++z) {
            const int64_t iz = (int64_t)tzi * p.tz + z;
            if (iz >= p.n_z) break;
            const float4 e = p.tab[row * p.n_a * p.n_z + ia * p.n_z + iz];
            bool ok = true;
            if (p.is_rx) ok = (p.mode == MODE_EXACT) ? (e.w > 0.0f) : (e.z != 0.0f);
            if (ok) { lo = fminf(lo, e.x); hi = fmaxf(hi, e.x); }
        }
    }
    p.out[i] = make_float2(lo, hi);
}

cudaError_t launch_range(const RangeParams &p, cudaStream_t st)
{
    const int64_t n = (int64_t)p.rows * p.tiles_a * p.tiles_z;
    if (n <= 0) return cudaSuccess;
    range_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(p);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------
// Mask: sum over receive elements of the apodisation, for every insonified
// (pixel, tx) (RCA.cu:247-250, 301-304), summed over transmits when
// compounding (RCA.m:696).
// ------------------------------------------------------------------------
__global__ void mask_kernel(const DevGeom g, float *mask, int compound, int accumulate)
{
    const int64_t n_vox = g.n_z * g.n_u * g.n_v;
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n_vox) return;
    const int64_t iz = v % g.n_z, iu = (v / g.n_z) % g.n_u, iv = v / (g.n_z * g.n_u);
    const int64_t rxkey = iu * g.n_z + iz, txkey = iv * g.n_z + iz;
    const int64_t pix = iz * g.s_z + iu * g.s_u + iv * g.s_v;
    const float a = g.apod_sum[rxkey];
    float total = 0.0f;
    for (int tx = 0; tx < g.n_tx; ++tx) {
        const float4 t = g.tx_tab[(int64_t)tx * g.n_v * g.n_z + txkey];
        bool cone = ((g.mode == MODE_EXACT) ? t.w : t.y) != 0.0f;
        if (g.cone_u) cone = cone && g.cone_u[(int64_t)tx * g.n_u * g.n_z + rxkey] != 0;
        const float m = cone ? a : 0.0f;
        if (compound) {
            total = __fadd_rn(total, m);
        } else {
            float *o = mask + (int64_t)tx * g.n_pix + pix;
            *o = accumulate ? *o + m : m;
        }
    }
    if (compound) mask[pix] = accumulate ? mask[pix] + total : total;
}

cudaError_t launch_mask(const DevGeom &g, float *mask, int compound, int accumulate, cudaStream_t st)
{
    const int64_t n = g.n_z * g.n_u * g.n_v;
    mask_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, mask, compound, accumulate);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------
// FP32 FMA throughput probe: 8 independent FMA chains per thread.
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(256) fma_probe_kernel(float *out, int iters, float b, float c)
{
    float a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = (float)(threadIdx.x + k) * 1e-3f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u)
#pragma unroll
            for (int k = 0; k < 8; ++k) a[k] = fmaf(a[k], b, c);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == 12345.678f) out[threadIdx.x] = s;  // keeps the chains live
}

cudaError_t launch_fma_probe(float *out, int blocks, int iters, cudaStream_t st)
{
    fma_probe_kernel<<<blocks, 256, 0, st>>>(out, iters, 0.999999f, 1e-6f);
    return cudaGetLastError();
}

}  // namespace rcabf
