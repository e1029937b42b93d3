// Fused + plain kernel instantiations: EXACT tables, kind K_LANCZOS4.
#include "fused_inst.cuh"
RCABF_EXACT_TU(K_LANCZOS4, exact_l4)
RCABF_VB_TU(K_LANCZOS4, exact_l4)
