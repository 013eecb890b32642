// Project-written stand-in for the absent driveless header of this name.
// Only what the FastRRT sources use: truncating TO_INT and double-precision
// angle constants (assumed; the real library is not available).
#pragma once
#ifndef TO_INT
#define TO_INT(x) static_cast<int>(x)
#endif
#ifndef PI
#define PI 3.14159265358979323846
#endif
#ifndef HALF_PI
#define HALF_PI (PI / 2.0)
#endif
#ifndef TO_DEG
#define TO_DEG (180.0 / PI)
#endif
#ifndef TO_RAD
#define TO_RAD (PI / 180.0)
#endif
