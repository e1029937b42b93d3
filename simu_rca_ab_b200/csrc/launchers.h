// Host-side launch entry points of the CUDA translation units.
#pragma once

#include <cuda_runtime.h>

#include "rcabf_internal.h"

namespace rcabf {

struct IngestParams {
    const void *iq;
    int32_t iq_dtype;
    int32_t n_sample, n_ele, n_tx;
    int64_t n_frame;
    int32_t fb, n_fb;
    void *S;
    int64_t slab_bytes;
    int32_t n_rows;        // rows written per slab: n_sample, or more with zero rows past the record
    void *S2;              // NULL, or a second slab set of the same layout holding (-im, re)
};

struct RangeParams {
    const float4 *tab;
    float2 *out;
    int64_t rows, n_a, n_z;
    int32_t ta, tz, tiles_a, tiles_z;
    int32_t mode, is_rx;
};

// Inputs of the REF_COMPAT table kernels: single-precision copies of what the
// reference wrapper hands its kernel (RCA.m:601-626), per table key.
struct RefTableParams {
    float4 *rx_tab;        // [n_ele][n_rxkey]
    float4 *tx_tab;        // [n_tx][n_txkey]
    uint8_t *cone_u;       // [n_tx][n_rxkey] or NULL
    float *apod_sum;       // [n_rxkey]
    const float *rx_key_u, *rx_key_z;   // per rx key
    const float *tx_key_v, *tx_key_z;   // per tx key
    const float *ele_u, *ele_z;         // per element (receive axis, depth)
    const float *vs_u, *vs_v, *vs_z;    // per tx, virtual source along u, v, z
    const float *min_dist;              // per tx
    int64_t n_rxkey, n_txkey;
    int32_t n_ele, n_tx;
    float half_ap_u, half_ap_v, ap_z;   // half apertures along u / v, aperture along z
    float fnumber, inv_c;
    int32_t receive_x;
    int32_t mask_transmit;
    float fd, fs;          // for the phase-rate ratio fdividef(fd, fs) (RCA.cu:372)
    float *ratio_out;      // one float
};

cudaError_t launch_ingest(const IngestParams &p, int store, cudaStream_t st);
cudaError_t launch_range(const RangeParams &p, cudaStream_t st);
cudaError_t launch_mask(const DevGeom &g, float *mask, int compound, int accumulate, cudaStream_t st);
cudaError_t launch_fma_probe(float *out, int blocks, int iters, cudaStream_t st);
cudaError_t launch_ref_tables(const RefTableParams &p, cudaStream_t st);

// Fused kernel (persistent).  kind: Kind, store: Store, fb in {1,2,4,8,16}.
cudaError_t launch_fused(int mode, int kind, int fb, int store, const FusedParams &p, int grid,
                         size_t smem, cudaStream_t st);
// Shared memory the fused kernel may use (opt-in beyond 48 KB), per variant.
cudaError_t prepare_fused(int mode, int kind, int fb, int store, size_t smem);
// Resident CTAs per SM for a variant at a given dynamic shared memory size.
int fused_occupancy(int mode, int kind, int fb, int store, size_t smem);

// Voxel-blocked fused kernel (EXACT tables): d = row shift bound (1 or 2),
// fb in {2, 4, 8, 16}; 128 threads per CTA; tm = 1: accumulators in tensor
// memory, occupancy capped by the SM's 512 TMEM columns.
cudaError_t launch_fused_vb(int kind, int d, int tm, int fb, int store, const FusedParams &p, int grid,
                            size_t smem, cudaStream_t st);
cudaError_t prepare_fused_vb(int kind, int d, int tm, int fb, int store, size_t smem);
int fused_vb_occupancy(int kind, int d, int tm, int fb, int store, size_t smem);

// Tensor-core kernel (FP16 slabs, EXACT tables, compounded output; one CTA
// per SM, all 512 tensor-memory columns): fb frames per block (multiple of
// 8, 32..tc_max_frames_per_block(split)), slabs of rows_per_slab rows of
// 2 fb halfs.  split = 1: weights as two FP16 terms (hi + remainder).
cudaError_t launch_fused_tc(int kind, int split, int bf16, const FusedJob &job, int fb, int rows_per_slab, int64_t n_items,
                            unsigned long long *err, int n_sm, cudaStream_t st);
int tc_max_frames_per_block(int split);
int tc_tmem_columns(int fb, int split);

// The current device's bound-check / timeout counter (allocated on first use;
// read and cleared by rcabf_take_error_count), and the library's count of
// kernel launches (rcabf_take_launch_count).
unsigned long long *current_error_counter();
void count_launches(int64_t n);
size_t tc_launch_smem(int fb);

// Plain kernel: one frame.
cudaError_t launch_plain(int mode, int kind, const PlainParams &p, cudaStream_t st);

// Device addresses, on the current device, of the static workspace
// (RCABF_NOALLOC_WORKSPACE_BYTES) and error counter of rcabf_beamform_noalloc.
cudaError_t noalloc_region(void **ws, unsigned long long **err);

}  // namespace rcabf
