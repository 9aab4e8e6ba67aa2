"""B200-native batched collision queries (RTCollisionDetection's detector path).

The engine is ``librtcd_b200.so`` (CUDA, sm_100a) behind the C ABI in
``include/rtcd.h``; :mod:`rtcollisiondetection_b200.rtcd` binds it.
"""
from . import scenes  # noqa: F401
