/*
 * helper_cuda.h -- project-written stand-in for the CUDA samples header the
 * reference includes (e.g. lbm.cu:27).  TEST INFRASTRUCTURE ONLY.  The step
 * modules use only checkCudaErrors, and cudaThreadSynchronize, which CUDA 12
 * keeps only as a deprecated alias of cudaDeviceSynchronize.
 */
#ifndef REF_HARNESS_HELPER_CUDA_H
#define REF_HARNESS_HELPER_CUDA_H
#include <stdio.h>
#include <stdlib.h>
#include <cuda_runtime.h>

#define checkCudaErrors(call)                                                          \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) {                                                       \
            fprintf(stderr, "CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
            exit(1);                                                                   \
        }                                                                              \
    } while (0)

#define cudaThreadSynchronize cudaDeviceSynchronize
#endif
