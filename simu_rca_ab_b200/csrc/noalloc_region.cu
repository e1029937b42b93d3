// Static device scratch of rcabf_beamform_noalloc: the fused path's
// workspace (ingested slabs + window-range tables) and its error counter
// live in file-scope device arrays, so that entry point allocates nothing.
// One copy per device (the module is loaded per context); overlapping calls
// on one device share it.
#include <cuda_runtime.h>

#include "../../include/rcabf.h"
#include "launchers.h"

namespace rcabf {

static __device__ __align__(256) unsigned char g_noalloc_ws[RCABF_NOALLOC_WORKSPACE_BYTES];
static __device__ __align__(8) unsigned long long g_noalloc_err;

cudaError_t noalloc_region(void **ws, unsigned long long **err)
{
    cudaError_t e = cudaGetSymbolAddress(ws, g_noalloc_ws);
    if (e != cudaSuccess) return e;
    return cudaGetSymbolAddress(reinterpret_cast<void **>(err), g_noalloc_err);
}

}  // namespace rcabf
