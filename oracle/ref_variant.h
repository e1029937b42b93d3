/*
 * oracle/ref_variant.h -- TEST INFRASTRUCTURE ONLY.
 *
 * Selects which reference kernel source the oracle harnesses include
 * (RCA_VARIANT, set by oracle/Makefile; each lives in its own directory of
 * the reference, put on the include path there):
 *   0  RCA/bfVirtualSourceGeneric_RCA.cu                 the beamformer
 *   1  Hyp1_save/bfVirtualSourceGeneric_RCA_ab_1.cu      + receive aberration law per element
 *   2  Hyp2/bfVirtualSourceGeneric_RCA_ab_2.cu           + receive aberration law per (transmit, element)
 *   3  NoSum/bfVirtualSourceGeneric_RCA_Nosum.cu         one output per receive element (no sum)
 *   4  NoSum_ab/bfVirtualSourceGeneric_RCA_Nosum_ab.cu   no sum + aberration law per element
 * The aberration variants take `const float *AbLawRx` after startTime
 * (..._ab_1.cu:124-125); RCA_AB_ARG inserts it in the call.
 */
#pragma once

#ifndef RCA_VARIANT
#define RCA_VARIANT 0
#endif

#if RCA_VARIANT == 0
#include "bfVirtualSourceGeneric_RCA.cu"
#define RCA_KERNEL bfVirtualSourceGeneric_RCA
#define RCA_HAS_AB 0
#elif RCA_VARIANT == 1
#include "bfVirtualSourceGeneric_RCA_ab_1.cu"
#define RCA_KERNEL bfVirtualSourceGeneric_RCA_ab_1
#define RCA_HAS_AB 1
#elif RCA_VARIANT == 2
#include "bfVirtualSourceGeneric_RCA_ab_2.cu"
#define RCA_KERNEL bfVirtualSourceGeneric_RCA_ab_2
#define RCA_HAS_AB 1
#elif RCA_VARIANT == 3
#include "bfVirtualSourceGeneric_RCA_Nosum.cu"
#define RCA_KERNEL bfVirtualSourceGeneric_RCA_Nosum
#define RCA_HAS_AB 0
#elif RCA_VARIANT == 4
#include "bfVirtualSourceGeneric_RCA_Nosum_ab.cu"
#define RCA_KERNEL bfVirtualSourceGeneric_RCA_Nosum_ab
#define RCA_HAS_AB 1
#else
#error "unknown RCA_VARIANT"
#endif

#if RCA_HAS_AB
#define RCA_AB_ARG abLaw,
#else
#define RCA_AB_ARG
#endif
