// All delay-and-sum kernels of librcabf.
#pragma once

#include "das_common.cuh"
#include "fused_kernel.cuh"
#include "plain_kernel.cuh"
