/*
 * oracle/ref_sim_harness.cpp -- TEST INFRASTRUCTURE ONLY (simulator oracle "O1").
 *
 * Runs the reference simulator kernels TXfield and RXfield, compiled from
 * their own unmodified source (MATLAB/lib/simulator/SimUS_CUDARCA.cu,
 * included below through the include path set by oracle/Makefile), on the
 * host cores.  Every CUDA thread of those kernels writes exactly one output
 * element from its own (frequency, scatterer, transmit) or (frequency,
 * element, scatterer) coordinates (SimUS_CUDARCA.cu:230-236, 318-324), so the
 * harness calls the kernel body once per coordinate with blockDim = 1 and
 * the coordinate in blockIdx; OpenMP spreads the calls over threads.
 *
 * cuComplex.h is included before the CUDA-to-host shim so that its own
 * helpers keep the host math they were written with; the kernels' CUDA math
 * calls go to the double-evaluated versions of refmath.h.
 */
#include <cuComplex.h>
#include "ref_shim.h"

#define expf   rm_expf
#define asinf  rm_asinf
#define atan2f rm_atan2f
#define sqrtf  rm_sqrtf
#define fabsf  rm_fabsf

#include "SimUS_CUDARCA.cu"

#include <omp.h>

extern "C" int sim_ref_cpu_txfield(
    cuFloatComplex *TX, const float *r_scat, const float *r_ele, const cuFloatComplex *k,
    const cuFloatComplex *pulse, const cuFloatComplex *ir, const float *delay, const float *apod,
    float width, float height, float rfocus, float baffle, float lens, float c,
    int nscat, int nele, int nf, int ntx, int nsub, int nthreads)
{
    if (nscat <= 0 || nele <= 0 || nf <= 0 || ntx <= 0 || nsub <= 0) return 1;
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    const long total = (long)nf * nscat * ntx;
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (long i = 0; i < total; ++i) {
        const unsigned ik = (unsigned)(i % nf), is = (unsigned)((i / nf) % nscat), it = (unsigned)(i / ((long)nf * nscat));
        blockDim = rm_dim3{1u, 1u, 1u};
        threadIdx = rm_dim3{0u, 0u, 0u};
        blockIdx = rm_dim3{ik, is, it};
        TXfield(TX, r_scat, r_ele, k, pulse, ir, delay, apod, width, height, rfocus, baffle, lens, c,
                nscat, nele, nf, ntx, nsub);
    }
    return 0;
}

extern "C" int sim_ref_cpu_rxfield(
    cuFloatComplex *RX, const float *r_scat, const float *r_ele, const cuFloatComplex *k,
    const cuFloatComplex *ir, float width, float height, float rfocus, float baffle, float lens, float c,
    int nscat, int nele, int nf, int nsub, int nthreads)
{
    if (nscat <= 0 || nele <= 0 || nf <= 0 || nsub <= 0) return 1;
    if (nthreads <= 0) nthreads = omp_get_max_threads();
    const long total = (long)nf * nele * nscat;
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (long i = 0; i < total; ++i) {
        const unsigned ik = (unsigned)(i % nf), ie = (unsigned)((i / nf) % nele), is = (unsigned)(i / ((long)nf * nele));
        blockDim = rm_dim3{1u, 1u, 1u};
        threadIdx = rm_dim3{0u, 0u, 0u};
        blockIdx = rm_dim3{ik, ie, is};
        RXfield(RX, r_scat, r_ele, k, ir, width, height, rfocus, baffle, lens, c, nscat, nele, nf, nsub);
    }
    return 0;
}
