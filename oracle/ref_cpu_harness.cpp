/*
 * oracle/ref_cpu_harness.cpp -- TEST INFRASTRUCTURE ONLY (oracle "O1").
 *
 * Runs a reference RCA kernel, compiled from its own unmodified source
 * (MATLAB/lib/beamformer/RCA/bfVirtualSourceGeneric_RCA.cu, or one of its
 * aberration-law / per-channel variants: ref_variant.h, selected by
 * oracle/Makefile), on the host cores.  The
 * launch geometry is the one the reference wrapper uses
 * (bfVirtualSourceGeneric_RCA.m:645-650): blocks of 1024 threads, grid
 * [ceil(nPix/1024), nTx, nFrame].  OpenMP spreads the blocks over threads;
 * each CUDA thread is one call of the kernel body.
 *
 * The reference kernel writes each (pixel, transmit, frame) output and each
 * (pixel, transmit) mask entry from exactly one CUDA thread
 * (bfVirtualSourceGeneric_RCA.cu:229-252, 301-304), so the blocks can run in
 * any order.
 */
#include "ref_shim.h"
#include "ref_variant.h"

#include <omp.h>

extern "C" int rca_ref_cpu_run(
    float *dataBf, float *mask, const float *data,
    const float *gridBfX, const float *gridBfY, const float *gridBfZ,
    const float *posEleX, const float *posEleY, const float *posEleZ,
    const float *vsX, const float *vsY, const float *vsZ,
    const float *minDist, int flagReceiveX,
    float apertureX, float apertureY, float apertureZ,
    float samplingFrequency, float demodulationFrequency, float speedOfSound,
    float startTime, const float *abLaw, float fnumber,
    int nPix, int nChannel, int nTx, int nFrame, int nSample,
    int flagLanczos, int flagMaskTransmit, int nThreads)
{
    if (nPix <= 0 || nChannel <= 0 || nTx <= 0 || nFrame <= 0 || nSample <= 0) return 1;
    if (RCA_HAS_AB && !abLaw) return 3;
    (void)abLaw;
    const int blk = 1024;
    const int gx = (nPix + blk - 1) / blk;
    const long nBlocks = (long)gx * nTx * nFrame;
    if (nThreads <= 0) nThreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nThreads)
    for (long b = 0; b < nBlocks; ++b) {
        const unsigned bx = (unsigned)(b % gx);
        const unsigned by = (unsigned)((b / gx) % nTx);
        const unsigned bz = (unsigned)(b / ((long)gx * nTx));
        blockIdx = rm_dim3{bx, by, bz};
        blockDim = rm_dim3{(unsigned)blk, 1u, 1u};
        for (unsigned t = 0; t < (unsigned)blk; ++t) {
            threadIdx = rm_dim3{t, 0u, 0u};
            RCA_KERNEL(
                dataBf, mask, data, gridBfX, gridBfY, gridBfZ,
                posEleX, posEleY, posEleZ, vsX, vsY, vsZ, minDist,
                flagReceiveX != 0, apertureX, apertureY, apertureZ,
                samplingFrequency, demodulationFrequency, speedOfSound,
                startTime, RCA_AB_ARG fnumber, nPix, nChannel, nTx, nFrame, nSample,
                flagLanczos != 0, flagMaskTransmit != 0);
        }
    }
    return 0;
}
