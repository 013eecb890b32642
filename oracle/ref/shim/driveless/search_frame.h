// Project-written stand-in: float3-per-pixel BEV frame (class id, distance
// to goal, traversability bits), its class-cost table and parameter slots.
#pragma once
#include <utility>
#include <vector>
#include "cuda_ptr.h"
#include "cuda_params.h"
#include "angle.h"
#include "waypoint.h"
class SearchFrame
{
    int _w, _h;
    CudaPtr<float3> _frame;
    CudaPtr<float> *_costs = nullptr;
    int _ncosts = 0;
    CudaPtr<int> _params;

public:
    SearchFrame(int w, int h, std::pair<int, int> lower, std::pair<int, int> upper)
        : _w(w), _h(h), _frame((size_t)w * h), _params(16)
    {
        int *p = _params.get();
        p[FRAME_PARAM_WIDTH] = w;
        p[FRAME_PARAM_HEIGHT] = h;
        p[FRAME_PARAM_CENTER_X] = w / 2;
        p[FRAME_PARAM_CENTER_Z] = h / 2;
        p[FRAME_PARAM_LOWER_BOUND_X] = lower.first;
        p[FRAME_PARAM_LOWER_BOUND_Z] = lower.second;
        p[FRAME_PARAM_UPPER_BOUND_X] = upper.first;
        p[FRAME_PARAM_UPPER_BOUND_Z] = upper.second;
    }
    ~SearchFrame() { delete _costs; }
    int width() { return _w; }
    int height() { return _h; }
    float3 *getCudaPtr() { return _frame.get(); }
    float *getCudaClassCostsPtr() { return _costs ? _costs->get() : nullptr; }
    int getClassCount() { return _ncosts; }
    int *getCudaFrameParamsPtr() { return _params.get(); }
    void setClassCosts(const std::vector<float> &c)
    {
        delete _costs;
        _costs = new CudaPtr<float>(c.size());
        for (size_t i = 0; i < c.size(); i++)
            _costs->get()[i] = c[i];
        _ncosts = (int)c.size();
    }
    // half footprint, stored as the planner stores it (already halved)
    void setHalfMinDistance(int mdx, int mdz)
    {
        _params.get()[FRAME_PARAM_MIN_DIST_X] = mdx;
        _params.get()[FRAME_PARAM_MIN_DIST_Z] = mdz;
    }
    void copyFrom(const float *xyz)
    {
        float3 *f = _frame.get();
        for (long i = 0; i < (long)_w * _h; i++)
            f[i] = make_float3(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    }
    bool isObstacle(int x, int z)
    {
        int c = TO_INT(_frame.get()[(long)z * _w + x].x);
        return getCudaClassCostsPtr()[c] < 0;
    }
    bool isSafeZoneChecked() { return false; }
    bool isDistanceToGoalProcessed() { return false; }
};
