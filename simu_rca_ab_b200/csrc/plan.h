// Launch plan of one beamform call: frame blocking, tile shape, shared-memory
// window size and workspace layout.
#pragma once

#include <cstddef>
#include <cstdint>

#include "geometry.h"

namespace rcabf {

// Shared memory the fused kernel may take per CTA (two CTAs fit an SM).
constexpr size_t SMEM_BUDGET = 110 * 1024;

struct Plan {
    int kernel = 0;       // rcabf_kernel
    int pc_all = 0;       // per-channel output, every frame in one launch (pc_das_kernel)
    int vb = 0;           // voxel-blocked kernel (fused_vb_kernel.cuh): 1 register, 2 TMEM accumulators
    int tc = 0;           // tensor-core kernel (fused_tc_kernel.cuh): 1 FP16 weights, 2 hi + remainder weights
    int tc_rows = 0;      // its slab rows (the record + zero rows a window may reach past it)
    int d = 0;            // its row shift bound
    int store = 0;
    int fb = 1, n_fb = 1;
    TileShape ts{1, 1, 256};
    int tiles_z = 0, tiles_u = 0, tiles_v = 0;
    int wmax = 0, row_words = 0;
    size_t smem = 0;
    int64_t slab_bytes = 0;
    size_t off_S = 0, off_rxr = 0, off_txr = 0, total = 0;
    int64_t n_items = 0;
};

// force: a launch choice to plan instead of the planner's own (autotuner);
// without one, a choice rcabf_autotune stored for these frames and storage
// is used.  RCABF_ERR_UNSUPPORTED when a forced choice does not fit.
int plan_beamform(rcabf_geometry *g, const rcabf_beamform_args *a, Plan &p, const TuneChoice *force = nullptr);

// Frame-block sizes with a compiled fused-kernel variant.
bool fb_supported(int mode, int fb);

// Shared-memory layout of the fused kernel (fused_kernel.cuh): the polyphase
// weight table (EXACT windowed-sinc kinds) followed by the window buffers --
// three for complex64 slabs (cp.async pipeline), two for FP16/BF16 slabs
// (register staging) -- each wmax rows of row_words 4-byte words.
inline int fused_stages(int store) { return store == ST_F32 ? 3 : 2; }
inline size_t fused_table_bytes(int mode, int kind) { return (mode == MODE_EXACT && kind != K_QUAD3) ? 16384 : 0; }
inline size_t fused_smem_bytes(int mode, int kind, int store, int wmax, int row_words)
{
    return fused_table_bytes(mode, kind) + (size_t)fused_stages(store) * wmax * row_words * 4;
}
// The voxel-blocked kernel keeps no table; three CTAs of 128 threads share an SM.
constexpr size_t VB_SMEM_BUDGET = 72 * 1024;
// 1: the planner gives the voxel-blocked kernel tensor-memory accumulators,
// 0: registers
constexpr int VB_TMEM_DEFAULT = 1;
// (with tensor-memory accumulators, vb = 2, followed by `zero_rows` staged
// rows of zeros that lanes without a contribution read)
inline size_t vb_smem_bytes(int store, int wmax, int row_words, int zero_rows = 0)
{
    return (size_t)(fused_stages(store) * wmax + zero_rows) * row_words * 4;
}
inline int vb_stage_rows_cap(int store, int fb)
{
    if (store == ST_F32) return 1 << 30;
    const int rawb = fb * 4, cs = rawb < 16 ? rawb : 16;
    return VB_STAGE_REGS * VB_THREADS_HOST / (rawb / cs);
}
// Staged rows are FP32 (8 bytes per frame), padded by 16 bytes when >= 16.
inline int fused_row_words(int fb) { return fb * 8 >= 16 ? (fb * 8 + 16) / 4 : (fb * 8) / 4; }
// Register staging holds at most 4 x 16-byte chunks per thread (256 threads).
inline int fused_stage_rows_cap(int store, int fb)
{
    if (store == ST_F32) return 1 << 30;
    const int rawb = fb * 4, cs = rawb < 16 ? rawb : 16;
    return 4 * 256 / (rawb / cs);
}

}  // namespace rcabf
