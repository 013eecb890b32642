// Project-written stand-in: a zero-initialised managed-memory array.
#pragma once
#include <cuda_runtime.h>
#include <cstring>
#include <memory>
#include "cuda_basic.h"
template <typename T>
class CudaPtr
{
    T *_p = nullptr;
    size_t _n = 0;

public:
    explicit CudaPtr(size_t n) : _n(n)
    {
        size_t cap = n < 16 ? 16 : n;
        if (cudaMallocManaged((void **)&_p, cap * sizeof(T)) != cudaSuccess)
            _p = nullptr;
        else
            memset((void *)_p, 0, cap * sizeof(T));
    }
    CudaPtr(const CudaPtr &) = delete;
    CudaPtr &operator=(const CudaPtr &) = delete;
    ~CudaPtr()
    {
        if (_p)
            cudaFree(_p);
    }
    T *get() { return _p; }
    size_t count() { return _n; }
};
template <typename T>
using cptr = std::unique_ptr<CudaPtr<T>>;
template <typename T>
using sptr = std::shared_ptr<CudaPtr<T>>;
