/*
 * ref_cpu_shim.h -- test infrastructure only (never linked into the product).
 *
 * Lets the reference's own CUDA C++ sources (main.cu, preprocess.cu,
 * fingerprint.cu, overlap.cu, scratch.cu) compile as a host program with
 * g++ and Thrust's OpenMP device system.  It maps the handful of CUDA
 * runtime calls the reference makes (cudaMalloc/cudaMallocHost/cudaFree/
 * cudaFreeHost/cudaMemcpy/cudaMemcpyToSymbol/cudaDeviceReset,
 * prelude.h:60-67, blocks.cuh:20-102, cqueue.cuh:65-151, main.cu:26,
 * fingerprint.cu:30-31, overlap.cu:120,245-246) onto host memory, and
 * erases the CUDA execution-space keywords so that every
 * `[] __host__ __device__ (...)` lambda becomes a plain lambda.
 *
 * The build recipe (oracle/Makefile, target `ref-cpu`) force-includes this
 * header plus the Thrust headers that Thrust 2.8 no longer pulls in
 * transitively.  No reference source is copied or modified.
 */
#ifndef EMP_REF_CPU_SHIM_H
#define EMP_REF_CPU_SHIM_H

#include <cstdlib>
#include <cstring>
#include <cassert>
#include <cerrno>
#include <cstdint>
#include <deque>
#include <vector>

#define __host__
#define __device__
#define __global__
#define __constant__
#define __forceinline__ inline

typedef int cudaError_t;
static const cudaError_t cudaSuccess = 0;
typedef enum {
    cudaMemcpyHostToHost = 0,
    cudaMemcpyHostToDevice = 1,
    cudaMemcpyDeviceToHost = 2,
    cudaMemcpyDeviceToDevice = 3,
    cudaMemcpyDefault = 4
} cudaMemcpyKind;

static inline const char *cudaGetErrorString(cudaError_t) { return "host shim"; }

static inline cudaError_t emp_shim_malloc(void **p, size_t n) {
    *p = std::malloc(n ? n : 1);
    return *p ? cudaSuccess : 2;
}
#define cudaMalloc(pp, n) emp_shim_malloc((void **)(pp), (n))
#define cudaMallocHost(pp, n) emp_shim_malloc((void **)(pp), (n))
static inline cudaError_t cudaFree(void *p) { std::free(p); return cudaSuccess; }
static inline cudaError_t cudaFreeHost(void *p) { std::free(p); return cudaSuccess; }
static inline cudaError_t cudaMemcpy(void *dst, const void *src, size_t n, cudaMemcpyKind) {
    if (n) std::memmove(dst, src, n);
    return cudaSuccess;
}
#define cudaMemcpyToSymbol(sym, src, n) (std::memcpy((void *)&(sym), (src), (n)), cudaSuccess)
static inline cudaError_t cudaDeviceReset() { return cudaSuccess; }

#endif
