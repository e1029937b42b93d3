/*
 * oracle/ref_shim.h -- TEST INFRASTRUCTURE ONLY.
 *
 * Lets the reference kernel source
 *   MATLAB/lib/beamformer/RCA/bfVirtualSourceGeneric_RCA.cu
 * compile unmodified as plain C++ for the CPU (oracle "O1").  The CUDA
 * qualifiers become nothing, the launch coordinates become thread-local
 * variables that the harness sets before calling the kernel body once per
 * CUDA thread, and the CUDA math functions the kernel calls are routed to the
 * double-evaluated versions in refmath.h.
 */
#ifndef RCABF_ORACLE_REF_SHIM_H
#define RCABF_ORACLE_REF_SHIM_H

#include <cmath>
#include <cstdlib>
#include "refmath.h"

struct rm_dim3 { unsigned x, y, z; };
static thread_local rm_dim3 blockIdx, threadIdx, blockDim;

/* abs(float) must resolve to the float overload, as it does in device code. */
using std::abs;

#define __global__
#define __device__
#define __constant__

#define sinpi    rm_sinpif
#define cospif   rm_cospif
#define fdividef rm_fdividef
#define norm3df  rm_norm3df
#define hypotf   rm_hypotf
#define cosf     rm_cosf
#define sinf     rm_sinf
#define acosf    rm_acosf
#define rsqrt    rm_rsqrt

#endif /* RCABF_ORACLE_REF_SHIM_H */
