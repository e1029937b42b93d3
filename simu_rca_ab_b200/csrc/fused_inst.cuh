// Explicit instantiation helpers for the fused and plain kernels.  Each
// instantiation translation unit includes this header and defines one entry
// point for one (mode, kind), so the many template variants compile in
// parallel.
#pragma once

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
    if (p.per_channel)
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

template <int KIND, int FB, int STORE, int D>
static cudaError_t vb_do(const FusedParams *p, int grid, size_t smem, cudaStream_t st, int what, int *occ)
{
    auto k = fused_vb_kernel<KIND, FB, STORE, D>;
    if (what == 1) return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (what == 2) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, k, VB_THREADS, smem);
    k<<<grid, VB_THREADS, smem, st>>>(*p);
    return cudaGetLastError();
}

template <int KIND, int STORE, int D>
static cudaError_t vb_fb(int fb, const FusedParams *p, int grid, size_t smem, cudaStream_t st, int what, int *occ)
{
    switch (fb) {
    case 2: return vb_do<KIND, 2, STORE, D>(p, grid, smem, st, what, occ);
    case 4: return vb_do<KIND, 4, STORE, D>(p, grid, smem, st, what, occ);
    case 8: return vb_do<KIND, 8, STORE, D>(p, grid, smem, st, what, occ);
    case 16: return vb_do<KIND, 16, STORE, D>(p, grid, smem, st, what, occ);
    default: return cudaErrorInvalidValue;
    }
}

template <int KIND, int D>
static cudaError_t vb_store(int store, int fb, const FusedParams *p, int grid, size_t smem, cudaStream_t st,
                            int what, int *occ)
{
    switch (store) {
    case ST_F32: return vb_fb<KIND, ST_F32, D>(fb, p, grid, smem, st, what, occ);
    case ST_F16: return vb_fb<KIND, ST_F16, D>(fb, p, grid, smem, st, what, occ);
    case ST_BF16: return vb_fb<KIND, ST_BF16, D>(fb, p, grid, smem, st, what, occ);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace rcabf

#define RCABF_VB_TU(KIND, NAME)                                                                      \
    namespace rcabf {                                                                                \
    cudaError_t vb_entry_##NAME(int d, int store, int fb, const FusedParams *p, int grid, size_t smem,\
                                cudaStream_t st, int what, int *occ)                                 \
    {                                                                                                \
        if (d == 1) return vb_store<KIND, 1>(store, fb, p, grid, smem, st, what, occ);               \
        if (d == 2) return vb_store<KIND, 2>(store, fb, p, grid, smem, st, what, occ);               \
        return cudaErrorInvalidValue;                                                                \
    }                                                                                                \
    }
