"""B200-native (sm_100a) rebuild of the HulkTracer ray-tracing hot path:
GPU SAH KD-tree build, KD traversal (full stack, short stack in registers or
shared memory, kd-restart, ropes), ray-triangle intersection and shading with
shadow rays, behind the C ABI in include/hulkcuda.h."""
from ._lib import (BUILD_BINNED, BUILD_LEARNED, BUILD_SAH_RESORT, BRUTE, FULLSTACK, ROPES, RESTART, RESTART_EARLY,  # noqa: F401
                   SHADE_CPU, SHADE_MIRROR, SHADE_PICTURE, SHORTSTACK, SMEMSTACK, VARIANTS, HkError)
from .engine import Context, KDTreeCUDA, TraceCUDA  # noqa: F401
