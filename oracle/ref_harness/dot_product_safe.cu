// dot_product_safe.cu -- replacement for the reference's dot_product.cu in the
// reference-kernel harness.  TEST INFRASTRUCTURE ONLY.
//
// The reference's reduction (dot_product.cu:12-71) finishes with a warp stage
// that calls __syncthreads() inside `if (tid < 32)` and reads shared memory
// without volatile, which is undefined behaviour on GPUs with independent
// thread scheduling.  This file provides the same two entry points with the
// same contract -- getNumBlocksAndThreads (dot_product.cu:171-189) and
// dot_product (dot_product.cu:192-223): the FP64 inner product of two device
// vectors of n elements, using at most `blocks` doubles of d_o as scratch and
// returning the value to the host -- with every barrier in uniform control
// flow.  Only the summation order differs from the reference.
#include <stdio.h>
#include <stdlib.h>
#include <cuda_runtime.h>

#include "def.h"

void getNumBlocksAndThreads(int n, int maxThreads, int &blocks, int &threads)
{
    threads = (n == 1) ? 1 : ((n < maxThreads * 2) ? n / 2 : maxThreads);
    if (threads < 1) threads = 1;
    blocks = n / (threads * 2);
    if (blocks < 1) blocks = 1;
}

#define DOT_THREADS 256

__global__ void dot_partial(const double *a, const double *b, double *out, int n, int per_block)
{
    __shared__ double s[DOT_THREADS];
    const int begin = blockIdx.x * per_block;
    const int end = min(n, begin + per_block);
    double v = 0.0;
    for (int i = begin + threadIdx.x; i < end; i += blockDim.x) v += a[i] * b[i];
    s[threadIdx.x] = v;
    __syncthreads();
    for (int w = DOT_THREADS / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = s[0];
}

__global__ void dot_final(double *buf, int m)
{
    __shared__ double s[DOT_THREADS];
    double v = 0.0;
    for (int i = threadIdx.x; i < m; i += blockDim.x) v += buf[i];
    s[threadIdx.x] = v;
    __syncthreads();
    for (int w = DOT_THREADS / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) buf[0] = s[0];
}

double dot_product(double *d_i1, double *d_i2, double *d_o, int n)
{
    int blocks, threads;
    getNumBlocksAndThreads(n, 256, blocks, threads);   // d_o holds `blocks` doubles (stress.cu:344-354)
    const int per_block = (n + blocks - 1) / blocks;
    dot_partial<<<blocks, DOT_THREADS>>>(d_i1, d_i2, d_o, n, per_block);
    dot_final<<<1, DOT_THREADS>>>(d_o, blocks);
    double r = 0.0;
    cudaMemcpy(&r, d_o, sizeof(double), cudaMemcpyDeviceToHost);
    return r;
}
