// Project-written stand-in: ego and search parameter builders.
#pragma once
#include <utility>
#include "angle.h"
#include "waypoint.h"
#include "search_frame.h"
class EgoParams
{
public:
    int _w = 0, _h = 0;
    std::pair<int, int> _lb{-1, -1}, _ub{-1, -1};
    float _maxCurv = -1, _pw = 1, _ph = 1, _len = 1;
    angle _steer;
    static EgoParams init(int w, int h) { EgoParams e; e._w = w; e._h = h; return e; }
    EgoParams &withEgoLowerBound(std::pair<int, int> v) { _lb = v; return *this; }
    EgoParams &withEgoUpperBound(std::pair<int, int> v) { _ub = v; return *this; }
    EgoParams &withMaxCurvature(float v) { _maxCurv = v; return *this; }
    EgoParams &withSearchPhysicalSize(float w, float h) { _pw = w; _ph = h; return *this; }
    EgoParams &withMaxSteeringAngle(angle a) { _steer = a; return *this; }
    EgoParams &withVehicleLength(float v) { _len = v; return *this; }
    EgoParams build() { return *this; }
    int width() { return _w; }
    int height() { return _h; }
    std::pair<float, float> searchFramePhysicalDimensions() { return {_pw, _ph}; }
    angle maxSteeringAngle() { return _steer; }
    float vehicleLength_m() { return _len; }
    float maxCurvature() { return _maxCurv; }
    std::pair<int, int> egoLowerBound() { return _lb; }
    std::pair<int, int> egoUpperBound() { return _ub; }
};
class SearchParams
{
public:
    Waypoint _s, _g;
    float _v = 1, _maxPath = 40, _tol = 20;
    int _timeout = -1;
    std::pair<int, int> _md{0, 0};
    angle _htol = angle::deg(10);
    SearchFrame *_frame = nullptr;
    static SearchParams init(Waypoint s, Waypoint g) { SearchParams p; p._s = s; p._g = g; return p; }
    SearchParams &withVelocity(float v) { _v = v; return *this; }
    SearchParams &withMinDistance(std::pair<int, int> v) { _md = v; return *this; }
    SearchParams &withTimeout(int v) { _timeout = v; return *this; }
    SearchParams &withMaxPathSize(float v) { _maxPath = v; return *this; }
    SearchParams &withDistanceToGoalTolerance(float v) { _tol = v; return *this; }
    SearchParams &withHeadingErrorTolerance(angle a) { _htol = a; return *this; }
    SearchParams &withFrame(SearchFrame *f) { _frame = f; return *this; }
    SearchParams build() { return *this; }
    SearchFrame *frame() { return _frame; }
    Waypoint start() { return _s; }
    Waypoint goal() { return _g; }
    float velocity_m_s() { return _v; }
    int timeout_ms() { return _timeout; }
    float maxPathSize_px() { return _maxPath; }
    float distanceToGoalTolerance_px() { return _tol; }
    angle headingErrorTolerance() { return _htol; }
    std::pair<int, int> minDistance() { return _md; }
};
