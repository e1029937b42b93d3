// Fused + plain kernel instantiations for REF_COMPAT tables (the reference's
// quadratic and 6-tap kernels, complex64 storage).  Compiled with
// -fmad=false so that no product is fused into a following addition.
#include "fused_inst.cuh"

namespace rcabf {

cudaError_t fused_entry_ref(int kind, int store, int fb, const FusedParams *p, int grid, size_t smem,
                            cudaStream_t st, int what, int *occ)
{
    if (store != ST_F32) return cudaErrorInvalidValue;
    if (kind == K_QUAD3) return fused_fb<MODE_REF, K_QUAD3, ST_F32>(fb, p, grid, smem, st, what, occ);
    if (kind == K_REF6) return fused_fb<MODE_REF, K_REF6, ST_F32>(fb, p, grid, smem, st, what, occ);
    return cudaErrorInvalidValue;
}

cudaError_t plain_entry_ref(int kind, const PlainParams &p, cudaStream_t st)
{
    if (kind == K_QUAD3) return plain_iq<MODE_REF, K_QUAD3>(p, st);
    if (kind == K_REF6) return plain_iq<MODE_REF, K_REF6>(p, st);
    return cudaErrorInvalidValue;
}

}  // namespace rcabf
