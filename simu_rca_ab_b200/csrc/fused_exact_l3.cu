// Fused + plain kernel instantiations: EXACT tables, kind K_LANCZOS3.
#include "fused_inst.cuh"
RCABF_EXACT_TU(K_LANCZOS3, exact_l3)
RCABF_VB_TU(K_LANCZOS3, exact_l3)
