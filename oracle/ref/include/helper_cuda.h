/* Stand-in for the CUDA-samples helper header that the reference program
 * includes (MCGPU-PET.h:173-176).  Only the three names the reference uses are
 * provided.  Test infrastructure: used solely to build the reference under
 * oracle/_ref, never by the product. */
#pragma once
#include <cstdio>
#include <cstdlib>
#include <cuda_runtime.h>

#define checkCudaErrors(call)                                                   \
  do {                                                                          \
    cudaError_t err_ = (call);                                                  \
    if (err_ != cudaSuccess) {                                                  \
      std::fprintf(stderr, "CUDA error '%s' at %s:%d\n",                        \
                   cudaGetErrorString(err_), __FILE__, __LINE__);               \
      std::exit(EXIT_FAILURE);                                                  \
    }                                                                           \
  } while (0)

#define getLastCudaError(msg)                                                   \
  do {                                                                          \
    cudaError_t err_ = cudaGetLastError();                                      \
    if (err_ != cudaSuccess) {                                                  \
      std::fprintf(stderr, "%s: %s\n", (msg), cudaGetErrorString(err_));        \
      std::exit(EXIT_FAILURE);                                                  \
    }                                                                           \
  } while (0)

static inline int gpuGetMaxGflopsDeviceId() { return 0; }
