// Project-written stand-in: a zero-initialised managed-memory W x H grid.
#pragma once
#include "cuda_ptr.h"
template <typename T>
class CudaFrame
{
    CudaPtr<T> _data;
    int _w, _h;

public:
    CudaFrame(int w, int h) : _data((size_t)w * h), _w(w), _h(h) {}
    T *getCudaPtr() { return _data.get(); }
    int width() { return _w; }
    int height() { return _h; }
};
