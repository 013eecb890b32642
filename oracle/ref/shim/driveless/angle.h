// Project-written stand-in: an angle held in radians (double).
#pragma once
#include <cmath>
#include "math_utils.h"
class angle
{
    double _r = 0;

public:
    angle() = default;
    static angle rad(double v) { angle a; a._r = v; return a; }
    static angle deg(double v) { angle a; a._r = v * TO_RAD; return a; }
    double rad() const { return _r; }
    double deg() const { return _r * TO_DEG; }
    bool operator==(const angle &o) const { return std::fabs(_r - o._r) < 1e-5; }
    bool operator!=(const angle &o) const { return !(*this == o); }
};
