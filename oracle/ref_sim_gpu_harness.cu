/*
 * oracle/ref_sim_gpu_harness.cu -- TEST INFRASTRUCTURE ONLY (simulator oracle "O2").
 *
 * The reference simulator kernels (MATLAB/lib/simulator/SimUS_CUDARCA.cu,
 * included unmodified).  The reference wrapper launches 128 x 8 blocks
 * (SimUS_CUDARCA.m: ThreadBlockSize [128 8 1]); built without fast math the
 * kernels need more registers than a 1024-thread block allows, so blocks
 * here are 128 x 2.  Each thread computes one output from its own
 * coordinates, so the block shape changes nothing else.
 */
#include <cuda_runtime.h>
#include "SimUS_CUDARCA.cu"

extern "C" int sim_ref_gpu_txfield(
    cuFloatComplex *TX, const float *r_scat, const float *r_ele, const cuFloatComplex *k,
    const cuFloatComplex *pulse, const cuFloatComplex *ir, const float *delay, const float *apod,
    float width, float height, float rfocus, float baffle, float lens, float c,
    int nscat, int nele, int nf, int ntx, int nsub, void *stream)
{
    if (nscat <= 0 || nele <= 0 || nf <= 0 || ntx <= 0 || nsub <= 0) return 1;
    dim3 block(128, 2, 1);
    dim3 grid((nf + 127) / 128, (nscat + 1) / 2, ntx);
    if (grid.y > 65535 || grid.z > 65535) return 2;
    TXfield<<<grid, block, 0, (cudaStream_t)stream>>>(TX, r_scat, r_ele, k, pulse, ir, delay, apod, width, height,
                                                     rfocus, baffle, lens, c, nscat, nele, nf, ntx, nsub);
    return (int)cudaGetLastError();
}

extern "C" int sim_ref_gpu_rxfield(
    cuFloatComplex *RX, const float *r_scat, const float *r_ele, const cuFloatComplex *k,
    const cuFloatComplex *ir, float width, float height, float rfocus, float baffle, float lens, float c,
    int nscat, int nele, int nf, int nsub, void *stream)
{
    if (nscat <= 0 || nele <= 0 || nf <= 0 || nsub <= 0) return 1;
    dim3 block(128, 2, 1);
    dim3 grid((nf + 127) / 128, (nele + 1) / 2, nscat);
    if (grid.y > 65535 || grid.z > 65535) return 2;
    RXfield<<<grid, block, 0, (cudaStream_t)stream>>>(RX, r_scat, r_ele, k, ir, width, height, rfocus, baffle, lens, c,
                                                     nscat, nele, nf, nsub);
    return (int)cudaGetLastError();
}
