// Fused + plain kernel instantiations: EXACT tables, kind K_REF6.
#include "fused_inst.cuh"
RCABF_EXACT_TU(K_REF6, exact_ref6)
RCABF_VB_TU(K_REF6, exact_ref6)
