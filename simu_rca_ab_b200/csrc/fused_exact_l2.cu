// Fused + plain kernel instantiations: EXACT tables, kind K_LANCZOS2.
#include "fused_inst.cuh"
RCABF_EXACT_TU(K_LANCZOS2, exact_l2)
RCABF_VB_TU(K_LANCZOS2, exact_l2)
