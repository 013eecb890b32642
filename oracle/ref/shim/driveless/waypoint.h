// Project-written stand-in: integer grid waypoint with a heading.
#pragma once
#include <cmath>
#include "angle.h"
class Waypoint
{
    int _x = 0, _z = 0;
    angle _h;

public:
    Waypoint() = default;
    Waypoint(int x, int z, angle h) : _x(x), _z(z), _h(h) {}
    int x() const { return _x; }
    int z() const { return _z; }
    angle heading() const { return _h; }
    static double distanceBetween(const Waypoint &a, const Waypoint &b)
    {
        double dx = b._x - a._x, dz = b._z - a._z;
        return std::sqrt(dx * dx + dz * dz);
    }
};
