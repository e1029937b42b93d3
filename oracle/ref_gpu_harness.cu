/*
 * oracle/ref_gpu_harness.cu -- TEST INFRASTRUCTURE ONLY (oracle "O2").
 *
 * The reference RCA kernel compiled from its own unmodified source
 * (MATLAB/lib/beamformer/RCA/bfVirtualSourceGeneric_RCA.cu, included through
 * the include path set by oracle/Makefile) for sm_100a, launched with the
 * reference wrapper's geometry (bfVirtualSourceGeneric_RCA.m:645-650).
 * oracle/Makefile builds this file three times:
 *   strict  : no fast math, no FMA contraction (source-order IEEE arithmetic)
 *   fast    : -use_fast_math, as the reference wrapper compiles it (.m:796)
 *   default : nvcc defaults
 * The caller passes device pointers and chunks frames so that the kernel's
 * 32-bit indices stay in range, as the wrapper does (.m:587-594).
 */
#include <cuda_runtime.h>
#include "ref_variant.h"

extern "C" int rca_ref_gpu_launch(
    float *dataBf, float *mask, const float *data,
    const float *gridBfX, const float *gridBfY, const float *gridBfZ,
    const float *posEleX, const float *posEleY, const float *posEleZ,
    const float *vsX, const float *vsY, const float *vsZ,
    const float *minDist, int flagReceiveX,
    float apertureX, float apertureY, float apertureZ,
    float samplingFrequency, float demodulationFrequency, float speedOfSound,
    float startTime, const float *abLaw, float fnumber,
    int nPix, int nChannel, int nTx, int nFrame, int nSample,
    int flagLanczos, int flagMaskTransmit, void *stream)
{
    if (nPix <= 0 || nChannel <= 0 || nTx <= 0 || nFrame <= 0 || nSample <= 0) return 1;
    if (nTx > 65535 || nFrame > 65535) return 2;
    dim3 block(1024, 1, 1);
    dim3 grid((nPix + 1023) / 1024, nTx, nFrame);
    if (RCA_HAS_AB && !abLaw) return 3;
    (void)abLaw;
    RCA_KERNEL<<<grid, block, 0, (cudaStream_t)stream>>>(
        dataBf, mask, data, gridBfX, gridBfY, gridBfZ,
        posEleX, posEleY, posEleZ, vsX, vsY, vsZ, minDist,
        flagReceiveX != 0, apertureX, apertureY, apertureZ,
        samplingFrequency, demodulationFrequency, speedOfSound,
        startTime, RCA_AB_ARG fnumber, nPix, nChannel, nTx, nFrame, nSample,
        flagLanczos != 0, flagMaskTransmit != 0);
    return (int)cudaGetLastError();
}
