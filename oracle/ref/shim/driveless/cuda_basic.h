// Project-written stand-in: error macro and zero-copy host allocation.
#pragma once
#include <cuda_runtime.h>
#include <cstdio>
#include <cstddef>
#include <string>
#include <stdexcept>
#include "cuda_params.h"
#define CUDA(x)                                                              \
    do {                                                                     \
        cudaError_t e_ = (x);                                                \
        if (e_ != cudaSuccess)                                               \
            fprintf(stderr, "[ref shim] CUDA error %s\n", cudaGetErrorString(e_)); \
    } while (0)
template <typename T>
inline bool cudaAllocMapped(T **ptr, size_t size)
{
    return cudaHostAlloc((void **)ptr, size, cudaHostAllocMapped) == cudaSuccess;
}
