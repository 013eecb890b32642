"""B200-native FastRRT: the reference planner's API over hand-written CUDA
kernels for sm_100a (libfastrrt_b200.so, C ABI in include/fastrrt_b200.h)."""
from ._lib import FastRRTError, lib  # noqa: F401
from .driveless import EgoParams, SearchFrame, SearchParams, Waypoint, angle  # noqa: F401
from .fastrrt import FastRRT  # noqa: F401
from .kernels import Candidates  # noqa: F401
from .batch import BatchPlanner, make_request  # noqa: F401
