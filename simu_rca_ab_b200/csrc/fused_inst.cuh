// Explicit instantiation helpers for the fused and plain kernels.  Each
// instantiation translation unit includes this header and defines one entry
// point for one (mode, kind), so the many template variants compile in
// parallel.
#pragma once

#include <algorithm>

#include "das_kernels.cuh"
#include "launchers.h"

namespace rcabf {

// what: 0 launch, 1 set the shared-memory attribute, 2 query occupancy.
template <int MODE, int KIND, int FB, int STORE>
static cudaError_t fused_do(const FusedParams *p, int grid, size_t smem, cudaStream_t st, int what, int *occ)
{
    auto k = fused_das_kernel<MODE, KIND, FB, STORE>;
    if (what == 1) return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (what == 2) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, k, FUSED_THREADS, smem);
    k<<<grid, FUSED_THREADS, smem, st>>>(*p);
    return cudaGetLastError();
}

template <int MODE, int KIND, int STORE>
static cudaError_t fused_fb(int fb, const FusedParams *p, int grid, size_t smem, cudaStream_t st, int what, int *occ)
{
    switch (fb) {
    case 1: return fused_do<MODE, KIND, 1, STORE>(p, grid, smem, st, what, occ);
    case 2: return fused_do<MODE, KIND, 2, STORE>(p, grid, smem, st, what, occ);
    case 4: return fused_do<MODE, KIND, 4, STORE>(p, grid, smem, st, what, occ);
    case 8: return fused_do<MODE, KIND, 8, STORE>(p, grid, smem, st, what, occ);
    case 16: return fused_do<MODE, KIND, 16, STORE>(p, grid, smem, st, what, occ);
    default: break;
    }
    if constexpr (MODE == MODE_EXACT) {   // wider frame blocks: exact tables only
        switch (fb) {
        case 24: return fused_do<MODE, KIND, 24, STORE>(p, grid, smem, st, what, occ);
        case 32: return fused_do<MODE, KIND, 32, STORE>(p, grid, smem, st, what, occ);
        case 40: return fused_do<MODE, KIND, 40, STORE>(p, grid, smem, st, what, occ);
        default: break;
        }
    }
    return cudaErrorInvalidValue;
}

template <int MODE, int KIND, int IQ>
static cudaError_t plain_do(const PlainParams &p, cudaStream_t st)
{
    const int64_t n = p.g.n_z * p.g.n_u * p.g.n_v;
    if (p.per_channel && p.frame < 0) {   // every frame in one launch
        int dev = 0, n_sm = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
        const int64_t blocks = std::min<int64_t>((n * p.g.n_ele + 255) / 256, (int64_t)n_sm * 16);
        pc_das_kernel<MODE, KIND, IQ><<<(unsigned)blocks, 256, 0, st>>>(p);
    } else if (p.per_channel)
        plain_das_kernel<MODE, KIND, IQ, true><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(p);
    else
        plain_das_kernel<MODE, KIND, IQ, false><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(p);
    return cudaGetLastError();
}

template <int MODE, int KIND>
static cudaError_t plain_iq(const PlainParams &p, cudaStream_t st)
{
    switch (p.iq_dtype) {
    case 0: return plain_do<MODE, KIND, 0>(p, st);
    case 1: return plain_do<MODE, KIND, 1>(p, st);
    case 2: return plain_do<MODE, KIND, 2>(p, st);
    case 3: return plain_do<MODE, KIND, 3>(p, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace rcabf

// Defines rcabf::fused_entry_<NAME>(store, fb, ...) for all three storage
// types and rcabf::plain_entry_<NAME>(...).
#define RCABF_EXACT_TU(KIND, NAME)                                                                  \
    namespace rcabf {                                                                               \
    cudaError_t fused_entry_##NAME(int store, int fb, const FusedParams *p, int grid, size_t smem,  \
                                   cudaStream_t st, int what, int *occ)                             \
    {                                                                                               \
        switch (store) {                                                                            \
        case ST_F32: return fused_fb<MODE_EXACT, KIND, ST_F32>(fb, p, grid, smem, st, what, occ);   \
        case ST_F16: return fused_fb<MODE_EXACT, KIND, ST_F16>(fb, p, grid, smem, st, what, occ);   \
        case ST_BF16: return fused_fb<MODE_EXACT, KIND, ST_BF16>(fb, p, grid, smem, st, what, occ); \
        default: return cudaErrorInvalidValue;                                                      \
        }                                                                                           \
    }                                                                                               \
    cudaError_t plain_entry_##NAME(const PlainParams &p, cudaStream_t st)                           \
    {                                                                                               \
        return plain_iq<MODE_EXACT, KIND>(p, st);                                                   \
    }                                                                                               \
    }

// ---- voxel-blocked kernel (fused_vb_kernel.cuh) ----
#include "fused_vb_kernel.cuh"

namespace rcabf {

// Resident CTAs per SM of a kernel that allocates tensor memory, from its
// registers, shared memory and TMEM columns.  (For the voxel-blocked kernel
// with TMEM accumulators the runtime's occupancy query answered one CTA per
// SM where its registers allowed three.)
template <typename K>
static cudaError_t tmem_kernel_occupancy(K k, int threads, size_t smem, int cols, int *occ)
{
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, k);
    if (e != cudaSuccess) return e;
    int dev = 0, regs_sm = 0, smem_sm = 0, thr_sm = 0, blk_sm = 0, smem_res = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
    cudaDeviceGetAttribute(&blk_sm, cudaDevAttrMaxBlocksPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&smem_res, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    const int warps = (threads + 31) / 32;
    const int regs_warp = (fa.numRegs * 32 + 255) / 256 * 256;   // allocated per warp, 256 at a time
    const size_t smem_cta = (smem + fa.sharedSizeBytes + smem_res + 127) / 128 * 128;
    int n = std::min(blk_sm, thr_sm / (warps * 32));
    n = std::min(n, regs_warp > 0 ? regs_sm / regs_warp / warps : n);
    n = std::min(n, (int)((size_t)smem_sm / smem_cta));
    n = std::min(n, 512 / cols);
    *occ = std::max(n, 0);
    return cudaSuccess;
}

template <int KIND, int FB, int STORE, int D, bool TM>
static cudaError_t vb_do(const FusedParams *p, int grid, size_t smem, cudaStream_t st, int what, int *occ)
{
    auto k = fused_vb_kernel<KIND, FB, STORE, D, TM>;
    if (what == 1) return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (what == 2) {
        if constexpr (TM) return tmem_kernel_occupancy(k, VB_THREADS, smem, vb_tmem_cols_host(FB), occ);
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, k, VB_THREADS, smem);
    }
    k<<<grid, VB_THREADS, smem, st>>>(*p);
    return cudaGetLastError();
}

// tm: accumulators in tensor memory (32 to 128 columns per CTA)
template <int KIND, int STORE, int D>
static cudaError_t vb_fb(int tm, int fb, const FusedParams *p, int grid, size_t smem, cudaStream_t st, int what,
                         int *occ)
{
    if (tm) {
        switch (fb) {
        case 2: return vb_do<KIND, 2, STORE, D, true>(p, grid, smem, st, what, occ);
        case 4: return vb_do<KIND, 4, STORE, D, true>(p, grid, smem, st, what, occ);
        case 8: return vb_do<KIND, 8, STORE, D, true>(p, grid, smem, st, what, occ);
        case 16: return vb_do<KIND, 16, STORE, D, true>(p, grid, smem, st, what, occ);
        default: return cudaErrorInvalidValue;
        }
    }
    switch (fb) {
    case 2: return vb_do<KIND, 2, STORE, D, false>(p, grid, smem, st, what, occ);
    case 4: return vb_do<KIND, 4, STORE, D, false>(p, grid, smem, st, what, occ);
    case 8: return vb_do<KIND, 8, STORE, D, false>(p, grid, smem, st, what, occ);
    case 16: return vb_do<KIND, 16, STORE, D, false>(p, grid, smem, st, what, occ);
    default: return cudaErrorInvalidValue;
    }
}

template <int KIND, int D>
static cudaError_t vb_store(int tm, int store, int fb, const FusedParams *p, int grid, size_t smem,
                            cudaStream_t st, int what, int *occ)
{
    switch (store) {
    case ST_F32: return vb_fb<KIND, ST_F32, D>(tm, fb, p, grid, smem, st, what, occ);
    case ST_F16: return vb_fb<KIND, ST_F16, D>(tm, fb, p, grid, smem, st, what, occ);
    case ST_BF16: return vb_fb<KIND, ST_BF16, D>(tm, fb, p, grid, smem, st, what, occ);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace rcabf

#define RCABF_VB_TU(KIND, NAME)                                                                      \
    namespace rcabf {                                                                                \
    cudaError_t vb_entry_##NAME(int d, int tm, int store, int fb, const FusedParams *p, int grid,    \
                                size_t smem, cudaStream_t st, int what, int *occ)                    \
    {                                                                                                \
        if (d == 1) return vb_store<KIND, 1>(tm, store, fb, p, grid, smem, st, what, occ);           \
        if (d == 2) return vb_store<KIND, 2>(tm, store, fb, p, grid, smem, st, what, occ);           \
        return cudaErrorInvalidValue;                                                                \
    }                                                                                                \
    }
