"""yarnball_b200: B200-native Stable Cosserat Rods substep behind the YarnBall::Sim API.

The engine is the CUDA library yarnball_b200/_lib/libyarnball_b200.so (C ABI declared in
include/yarnball_b200.h).  This package is the Python mirror of YarnBall::Sim over that ABI.
"""
from ._abi import YarnBallError, load  # noqa: F401
from .sim import (MAX_COLLISIONS_PER_SEGMENT, Sim, VertexFlags, buildFromJSON, readFromBCC,  # noqa: F401
                  readFromOBJ, readFromPoly, resampleCMR, sort_pairs)
