// Launch plan of one beamform call: frame blocking, tile shape, shared-memory
// window size and workspace layout.
#pragma once

#include <cstddef>
#include <cstdint>

#include "geometry.h"

namespace rcabf {

// Shared memory the fused kernel's window buffers may take per CTA.
constexpr size_t SMEM_BUDGET = 96 * 1024;

struct Plan {
    int kernel = 0;       // rcabf_kernel
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

int plan_beamform(rcabf_geometry *g, const rcabf_beamform_args *a, Plan &p);

}  // namespace rcabf
