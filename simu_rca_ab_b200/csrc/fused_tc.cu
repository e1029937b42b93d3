// Tensor-core delay-and-sum kernel (fused_tc_kernel.cuh): instantiations,
// the slab tensor map and the launch.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

#include "fused_tc_kernel.cuh"
#include "launchers.h"

namespace rcabf {

// cuTensorMapEncodeTiled from the driver, looked up once through the
// runtime (no link-time dependency on libcuda).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

template <int KIND, bool SPLIT, bool BF>
static cudaError_t tc_do(const TcParams *p, int grid, size_t smem, cudaStream_t st, int what)
{
    auto k = fused_tc_kernel<KIND, SPLIT, BF>;
    if (what == 1) return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k<<<grid, TC_THREADS, smem, st>>>(*p);
    return cudaGetLastError();
}

// FP16 slabs with either weight precision; BF16 slabs with hi + remainder
// weights only
template <int KIND>
static cudaError_t tc_split(bool split, bool bf, const TcParams *p, int grid, size_t smem, cudaStream_t st, int what)
{
    if (bf) return split ? tc_do<KIND, true, true>(p, grid, smem, st, what) : cudaErrorInvalidValue;
    return split ? tc_do<KIND, true, false>(p, grid, smem, st, what) : tc_do<KIND, false, false>(p, grid, smem, st, what);
}

static cudaError_t tc_route(int kind, bool split, bool bf, const TcParams *p, int grid, size_t smem, cudaStream_t st,
                            int what)
{
    switch (kind) {
    case K_QUAD3: return tc_split<K_QUAD3>(split, bf, p, grid, smem, st, what);
    case K_REF6: return tc_split<K_REF6>(split, bf, p, grid, smem, st, what);
    case K_LANCZOS2: return tc_split<K_LANCZOS2>(split, bf, p, grid, smem, st, what);
    case K_LANCZOS3: return tc_split<K_LANCZOS3>(split, bf, p, grid, smem, st, what);
    case K_LANCZOS4: return tc_split<K_LANCZOS4>(split, bf, p, grid, smem, st, what);
    default: return cudaErrorInvalidValue;
    }
}

size_t tc_launch_smem(int fb)
{
    // at least half of an SM's shared memory, so that one CTA holds an SM
    // (the kernel allocates all 512 tensor-memory columns)
    return std::max<size_t>(tc_smem_bytes(fb), 116 * 1024);
}

int tc_max_frames_per_block(int split) { return tc_max_fb(split != 0); }
int tc_tmem_columns(int fb, int split) { return tc_tmem_cols(fb, split != 0); }

cudaError_t launch_fused_tc(int kind, int split, int bf16, const FusedJob &job, int fb, int rows_per_slab,
                            int64_t n_items, unsigned long long *err, int n_sm, cudaStream_t st)
{
    if (bf16 && !split) return cudaErrorInvalidValue;
    if (fb < 32 || fb > tc_max_fb(split != 0) || (fb & 7) || tc_tmem_cols(fb, split != 0) > 512)
        return cudaErrorInvalidValue;
    const int64_t rows = (int64_t)job.g.n_tx * job.g.n_ele * job.n_fb * rows_per_slab;   // of each slab set
    if (2 * rows >= ((int64_t)1 << 31)) return cudaErrorInvalidValue;
    auto enc = tensor_map_encoder();
    if (!enc) return cudaErrorNotSupported;
    TcParams p{};
    p.job = job;
    p.fb = fb;
    p.rows_per_slab = rows_per_slab;
    p.s2_row0 = rows;
    p.n_items = n_items;
    p.err_count = err;
    // the two slab sets (samples, then (-im, re)) as one 3-D FP16 tensor:
    // x = element within a 64-element
    // panel of a row (2-byte stride), y = row (rows of 2 fb halfs), z = panel
    // (128-byte stride); one box = one 16-row chunk of every panel, laid out
    // panel after panel with the 128-byte swizzle (the MMA's B layout).  The
    // last panel reaches past the row end into the next row: those columns
    // (>= 2 fb) are never read by the MMA, and the zero rows after each
    // record keep every read inside the slabs (a window ends at least one
    // row before its slab does).
    const int np = tc_panels(fb);
    cuuint64_t dims[3] = {64, (cuuint64_t)(2 * rows), (cuuint64_t)np};
    cuuint64_t strides[2] = {(cuuint64_t)(4 * fb), 128};
    cuuint32_t box[3] = {64, 16, (cuuint32_t)np};
    cuuint32_t es[3] = {1, 1, 1};
    const CUresult cr = enc(&p.tmap, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3, const_cast<void *>(job.S), dims, strides, box,
                            es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return cudaErrorInvalidValue;
    const size_t smem = tc_launch_smem(fb);
    if (job.g.mode != MODE_EXACT || !job.compound) return cudaErrorInvalidValue;
    cudaError_t e;
    if ((e = tc_route(kind, split != 0, bf16 != 0, nullptr, 0, smem, nullptr, 1)) != cudaSuccess) return e;
    const int grid = (int)std::min<int64_t>(n_items, n_sm);
    if (grid <= 0) return cudaSuccess;
    return tc_route(kind, split != 0, bf16 != 0, &p, grid, smem, st, 0);
}

}  // namespace rcabf
