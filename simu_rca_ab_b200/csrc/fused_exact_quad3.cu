// Fused + plain kernel instantiations: EXACT tables, kind K_QUAD3.
#include "fused_inst.cuh"
RCABF_EXACT_TU(K_QUAD3, exact_quad3)
RCABF_VB_TU(K_QUAD3, exact_quad3)
