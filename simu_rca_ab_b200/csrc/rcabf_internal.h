// Internal structures shared by the host code and the CUDA kernels of librcabf.
//
// Data layout in HBM (one geometry):
//   rx_tab  float4 [n_ele][n_rxkey]   rx key = iu * n_z + iz (u = receive axis)
//             EXACT      : {irx, ar, ai, apod}   irx = fs * tau_rx (samples, FP64-built),
//                                                (ar, ai) = apod * exp(+j 2 pi fd/fs irx)
//             REF_COMPAT : {delay_rx (s), apod, valid, 0}   reference FP32 arithmetic
//   tx_tab  float4 [n_tx][n_txkey]    tx key = iv * n_z + iz (v = transmit steering axis)
//             EXACT      : {itx, pr, pi, cone_v}  itx = fs * (tau_tx + t0),
//                                                 (pr, pi) = exp(+j 2 pi (fd/fs itx - 2 fd z / c))
//             REF_COMPAT : {delay_tx (s), cone_v, z (m, FP32), 0}
//   cone_u  uint8  [n_tx][n_rxkey]    transmit-cone test along the receive axis (or NULL)
//   apod_sum float [n_rxkey]          sum over elements of the apodisation (the reference's mask)
//   ab      float  [n_ele] or [n_tx][n_ele]  receive aberration delay (EXACT: samples, REF: s)
//   ab_ph   float2 same shape             EXACT only: exp(+j 2 pi fd ab)
// Channel data after ingest (workspace):
//   S       [tx][ele][frame block][sample][frame in block], storage type
//           (complex64, half2 or bf16x2), each (tx, ele, block) slab padded to 16 B.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define RCABF_HD __host__ __device__
#else
#define RCABF_HD
#endif

namespace rcabf {

enum Mode : int { MODE_EXACT = 0, MODE_REF = 1 };

// Interpolation kernels as compile-time kinds.  TAPS taps on samples
// n0 - LO .. n0 - LO + TAPS - 1; a sample index n0 is usable when
// LO <= n0 < n_sample - 1 - HI (the reference's rule, RCA.cu:233-243, 323).
enum Kind : int { K_QUAD3 = 0, K_REF6 = 1, K_LANCZOS2 = 2, K_LANCZOS3 = 3, K_LANCZOS4 = 4 };

template <int KIND> struct KindTraits;
template <> struct KindTraits<K_QUAD3>    { static constexpr int TAPS = 3, LO = 1, HI = 1, WIN = 0; };
template <> struct KindTraits<K_REF6>     { static constexpr int TAPS = 6, LO = 2, HI = 3, WIN = 2; };
template <> struct KindTraits<K_LANCZOS2> { static constexpr int TAPS = 4, LO = 1, HI = 2, WIN = 2; };
template <> struct KindTraits<K_LANCZOS3> { static constexpr int TAPS = 6, LO = 2, HI = 3, WIN = 3; };
template <> struct KindTraits<K_LANCZOS4> { static constexpr int TAPS = 8, LO = 3, HI = 4, WIN = 4; };

inline RCABF_HD int kind_lo(int k) { return k == K_QUAD3 ? 1 : k == K_LANCZOS2 ? 1 : k == K_LANCZOS4 ? 3 : 2; }
inline RCABF_HD int kind_hi(int k) { return k == K_QUAD3 ? 1 : k == K_LANCZOS2 ? 2 : k == K_LANCZOS4 ? 4 : 3; }
inline RCABF_HD int kind_taps(int k) { return k == K_QUAD3 ? 3 : k == K_LANCZOS2 ? 4 : k == K_LANCZOS4 ? 8 : 6; }

enum Store : int { ST_F32 = 0, ST_F16 = 1, ST_BF16 = 2 };
inline RCABF_HD int store_bytes(int st) { return st == ST_F32 ? 8 : 4; }

// Scalars the REF_COMPAT arithmetic needs, exactly as the reference kernel
// holds them (RCA.cu:121-125, 164, 372).
struct RefScalars {
    float fs, fd, t0, inv_c, ratio;  // ratio = fdividef(fd, fs)
};

// Device view of one geometry.
struct DevGeom {
    const float4 *rx_tab;
    const float4 *tx_tab;
    const uint8_t *cone_u;     // NULL when the transmit mask is off
    const float *apod_sum;
    const float *ab;           // NULL when no aberration law
    const float2 *ab_ph;       // EXACT only
    const float *wtab;         // EXACT windowed-sinc kinds: polyphase weight table (WT_Q x 16 floats)
    int32_t ab_per_tx;
    int32_t mode;
    int32_t n_ele, n_tx;
    int64_t n_z, n_u, n_v;     // tile space: rx key = iu*n_z+iz, tx key = iv*n_z+iz
    int64_t s_z, s_u, s_v;     // output pixel index strides
    int64_t n_pix;
    RefScalars ref;
};

// One acquisition inside a fused launch.
struct FusedJob {
    DevGeom g;
    const void *S;             // ingested channel data
    int64_t slab_bytes;        // bytes of one (tx, ele, block) slab
    const float2 *rx_range;    // [n_ele][tiles_u][tiles_z] (min, max) table delay per tile
    const float2 *tx_range;    // [n_tx][tiles_v][tiles_z]
    float2 *out;               // [frame][compound ? 1 : n_tx][pix]
    int64_t item_begin;        // first work item of this job
    int32_t n_fb, n_frame, n_sample;
    int32_t compound, accumulate;
    int32_t tiles_z, tiles_u, tiles_v;
    int32_t tu, tv, tz;        // tile shape, tu*tv*tz = blockDim.x
};

// Tensor-core kernel (fused_tc_kernel.cuh): voxel tiles of 128 voxels, tu
// (receive axis) x tv (steering axis) x 1 depth, with windows of at most
// TC_MAX_ROWS sample rows per (tx, rx) step; TC_TILE_U x TC_TILE_V is the
// preferred shape.
constexpr int TC_TILE_U = 4, TC_TILE_V = 32, TC_MAX_ROWS = 32;

constexpr int MAX_JOBS = 24;
constexpr int FUSED_THREADS = 256;
constexpr int FUSED_STAGES = 3;
constexpr int VB_BLOCK = 4;          // voxels per thread along v in the voxel-blocked kernel
constexpr int VB_THREADS_HOST = 128; // its CTA size
constexpr int VB_STAGE_REGS = 2;     // 16-byte staging chunks a thread holds (FP16/BF16 slabs)
constexpr int VB_MIN_BLOCKS = 1;     // launch-bounds hint: more forces spills (~230 registers live)
constexpr int VB_TM_MIN_BLOCKS = 4;  // the same with the accumulators in tensor memory (128 registers, no spills)
// tensor-memory columns a CTA of the voxel-blocked kernel allocates: 16 per
// frame pair, a power of two >= 32
constexpr RCABF_HD int vb_tmem_cols_host(int fb) { return fb * 8 <= 32 ? 32 : fb * 8; }

struct FusedParams {
    FusedJob jobs[MAX_JOBS];
    int32_t n_jobs;
    int32_t wmax;               // rows per shared-memory stage
    int32_t row_words;          // shared-memory row stride (4-byte words)
    int64_t n_items;
    unsigned long long *err_count;
};

// Plain kernel: one launch per frame, thread per voxel, global gathers from
// the caller's [frame][tx][ele][sample] layout.
struct PlainParams {
    DevGeom g;
    const void *iq;
    int32_t iq_dtype;           // rcabf_iq_dtype
    int32_t n_sample;
    int64_t frame;
    int64_t n_frame;
    int32_t compound, accumulate;
    int32_t per_channel;        // out is [element][frame][tx][pix]: one value per receive element
    float2 *out;
    unsigned long long *err_count;
};

}  // namespace rcabf
