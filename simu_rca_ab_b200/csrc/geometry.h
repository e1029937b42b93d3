// Host-side geometry object of librcabf: validated acquisition description,
// the derived virtual sources, and the device-resident delay tables.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/rcabf.h"
#include "rcabf_internal.h"

namespace rcabf {

struct TileShape {
    int tu, tv, tz;
    bool operator<(const TileShape &o) const
    {
        return std::array<int, 3>{tu, tv, tz} < std::array<int, 3>{o.tu, o.tv, o.tz};
    }
};

// A launch choice the autotuner can force on the planner: kernel family,
// frame block and tile shape (voxel-blocked: tv counts voxel blocks).
struct TuneChoice {
    int vb = 0;
    int fb = 0;
    TileShape ts{0, 0, 0};
    int tc = 0;       // tensor-core kernel: 1 single FP16 weights, 2 hi + remainder weights
};

// Spread of the table delay inside the tiles of one shape, used to size the
// shared-memory window (see window_rows()).
struct TileSpread {
    std::vector<float> tx_spread;  // per tile-z: max over (tx, tile-v) of max-min
    std::vector<float> rx_spread;  // per tile-z: max over (ele, tile-u) of max-min
};

}  // namespace rcabf

struct rcabf_geometry {
    int device = 0;
    int mode = 0;          // rcabf::Mode
    int interp = 0, lanczos_a = 0, kind = 0;
    int receive_x = 1, mask_transmit = 0;
    int grid_kind = 0;
    int64_t n_z = 0, n_u = 0, n_v = 0, s_z = 0, s_u = 0, s_v = 0, n_pix = 0;
    int n_ele = 0, n_tx = 0;
    double fs = 0, fd = 0, c = 0, t0 = 0, fnumber = 0;
    double ap_x = 0, ap_y = 0, ap_z = 0;
    std::vector<double> vs_x, vs_y, vs_z, min_dist;
    int has_ab = 0, ab_per_tx = 0;

    // host copies of the table delays (x component) for window sizing
    std::vector<float> rx_delay;   // [n_ele][n_rxkey], NaN where invalid
    std::vector<float> tx_delay;   // [n_tx][n_txkey]
    std::vector<float> ab_host;    // [n_ele] or [n_tx][n_ele] in table units

    // device buffers (owned)
    float4 *rx_tab = nullptr;
    float4 *tx_tab = nullptr;
    uint8_t *cone_u = nullptr;
    float *apod_sum = nullptr;
    float *ab = nullptr;
    float2 *ab_ph = nullptr;
    float *wtab = nullptr;
    rcabf::RefScalars ref{};

    std::mutex mu;
    std::map<rcabf::TileShape, rcabf::TileSpread> spreads;

    rcabf::DevGeom dev() const;
    // Upper bound of the window rows any tile of this shape needs for one
    // (tx, ele) step: spread of the transmit delay + spread of the receive
    // delay inside the tile (in samples) + the taps + rounding slack.
    int window_rows(const rcabf::TileShape &ts);
    // Tensor-core kernel: the 16-row window chunks its producer issues for
    // one frame block over all tiles of this shape and all (tx, element)
    // steps -- the same window arithmetic as the kernel, on the host copies
    // of the table delays -- i.e. its MMA work (each chunk is NMAT MMAs of
    // 128 x 2 FB x 16).
    int64_t tc_chunks(const rcabf::TileShape &ts, int64_t n_sample);
    std::map<std::array<int64_t, 3>, int64_t> tc_chunk_counts;
    // Largest difference of floor(sample index) between voxels of one
    // aligned block of `block` consecutive v (same u, z, tx, rx), i.e. the
    // row shift bound D of the voxel-blocked kernel; -1 if not applicable.
    int vb_shift(int block);
    std::map<int, int> vb_shifts;
    // launch choices found by rcabf_autotune, keyed by (frames, storage)
    std::map<std::array<int64_t, 2>, rcabf::TuneChoice> tuned;
};

namespace rcabf {
int build_geometry(const rcabf_geometry_desc *d, cudaStream_t st, rcabf_geometry **out);
void free_geometry(rcabf_geometry *g);
}  // namespace rcabf
