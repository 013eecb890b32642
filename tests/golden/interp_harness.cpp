// Runs the reference's own interpolate() (src/interpolation.cpp, compiled
// beside this file by make_interpolation.py) on control points read from
// stdin: "W H n" then n lines "x z heading"; prints the point count and
// "x z heading" per interpolated point (heading as a float, 9 digits).
#include <cstdio>
#include <vector>

#include "driveless/waypoint.h"

std::vector<Waypoint> interpolate(std::vector<Waypoint> &controlPoints, int width, int height);

int main()
{
    int W, H, n;
    if (std::scanf("%d %d %d", &W, &H, &n) != 3)
        return 2;
    std::vector<Waypoint> cps;
    for (int k = 0; k < n; k++) {
        int x, z;
        float h;
        if (std::scanf("%d %d %f", &x, &z, &h) != 3)
            return 2;
        cps.push_back(Waypoint(x, z, angle::rad(h)));
    }
    std::vector<Waypoint> out = interpolate(cps, W, H);
    std::printf("%zu\n", out.size());
    for (const Waypoint &w : out)
        std::printf("%d %d %.9g\n", w.x(), w.z(), (float)w.heading().rad());
    return 0;
}
