// Routes (mode, kind) to the instantiation translation unit that holds the
// kernel variant.
#include "launchers.h"

namespace rcabf {

#define DECL(NAME)                                                                                   \
    cudaError_t fused_entry_##NAME(int store, int fb, const FusedParams *p, int grid, size_t smem,   \
                                   cudaStream_t st, int what, int *occ);                             \
    cudaError_t plain_entry_##NAME(const PlainParams &p, cudaStream_t st);
DECL(exact_quad3)
DECL(exact_ref6)
DECL(exact_l2)
DECL(exact_l3)
DECL(exact_l4)
#undef DECL
cudaError_t fused_entry_ref(int kind, int store, int fb, const FusedParams *p, int grid, size_t smem,
                            cudaStream_t st, int what, int *occ);
cudaError_t plain_entry_ref(int kind, const PlainParams &p, cudaStream_t st);

#define DECL_VB(NAME)                                                                                \
    cudaError_t vb_entry_##NAME(int d, int tm, int store, int fb, const FusedParams *p, int grid,    \
                                size_t smem, cudaStream_t st, int what, int *occ);
DECL_VB(exact_quad3)
DECL_VB(exact_ref6)
DECL_VB(exact_l2)
DECL_VB(exact_l3)
DECL_VB(exact_l4)
#undef DECL_VB

static cudaError_t vb_route(int kind, int d, int tm, int fb, int store, const FusedParams *p, int grid,
                            size_t smem, cudaStream_t st, int what, int *occ)
{
    switch (kind) {
    case K_QUAD3: return vb_entry_exact_quad3(d, tm, store, fb, p, grid, smem, st, what, occ);
    case K_REF6: return vb_entry_exact_ref6(d, tm, store, fb, p, grid, smem, st, what, occ);
    case K_LANCZOS2: return vb_entry_exact_l2(d, tm, store, fb, p, grid, smem, st, what, occ);
    case K_LANCZOS3: return vb_entry_exact_l3(d, tm, store, fb, p, grid, smem, st, what, occ);
    case K_LANCZOS4: return vb_entry_exact_l4(d, tm, store, fb, p, grid, smem, st, what, occ);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_fused_vb(int kind, int d, int tm, int fb, int store, const FusedParams &p, int grid,
                            size_t smem, cudaStream_t st)
{
    return vb_route(kind, d, tm, fb, store, &p, grid, smem, st, 0, nullptr);
}

cudaError_t prepare_fused_vb(int kind, int d, int tm, int fb, int store, size_t smem)
{
    return vb_route(kind, d, tm, fb, store, nullptr, 0, smem, nullptr, 1, nullptr);
}

int fused_vb_occupancy(int kind, int d, int tm, int fb, int store, size_t smem)
{
    int occ = 0;
    if (vb_route(kind, d, tm, fb, store, nullptr, 0, smem, nullptr, 2, &occ) != cudaSuccess) return 0;
    return occ;
}

static cudaError_t fused_route(int mode, int kind, int fb, int store, const FusedParams *p, int grid,
                               size_t smem, cudaStream_t st, int what, int *occ)
{
    if (mode == MODE_REF) return fused_entry_ref(kind, store, fb, p, grid, smem, st, what, occ);
    switch (kind) {
    case K_QUAD3: return fused_entry_exact_quad3(store, fb, p, grid, smem, st, what, occ);
    case K_REF6: return fused_entry_exact_ref6(store, fb, p, grid, smem, st, what, occ);
    case K_LANCZOS2: return fused_entry_exact_l2(store, fb, p, grid, smem, st, what, occ);
    case K_LANCZOS3: return fused_entry_exact_l3(store, fb, p, grid, smem, st, what, occ);
    case K_LANCZOS4: return fused_entry_exact_l4(store, fb, p, grid, smem, st, what, occ);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_fused(int mode, int kind, int fb, int store, const FusedParams &p, int grid,
                         size_t smem, cudaStream_t st)
{
    return fused_route(mode, kind, fb, store, &p, grid, smem, st, 0, nullptr);
}

cudaError_t prepare_fused(int mode, int kind, int fb, int store, size_t smem)
{
    return fused_route(mode, kind, fb, store, nullptr, 0, smem, nullptr, 1, nullptr);
}

int fused_occupancy(int mode, int kind, int fb, int store, size_t smem)
{
    int occ = 0;
    if (fused_route(mode, kind, fb, store, nullptr, 0, smem, nullptr, 2, &occ) != cudaSuccess) return 0;
    return occ;
}

cudaError_t launch_plain(int mode, int kind, const PlainParams &p, cudaStream_t st)
{
    if (mode == MODE_REF) return plain_entry_ref(kind, p, st);
    switch (kind) {
    case K_QUAD3: return plain_entry_exact_quad3(p, st);
    case K_REF6: return plain_entry_exact_ref6(p, st);
    case K_LANCZOS2: return plain_entry_exact_l2(p, st);
    case K_LANCZOS3: return plain_entry_exact_l3(p, st);
    case K_LANCZOS4: return plain_entry_exact_l4(p, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace rcabf
