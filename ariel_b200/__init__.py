"""B200-native FLIP step of betajippity/Ariel: sm_100a CUDA kernels behind a C ABI.

The Python modules mirror the reference's FlipSim interface over that ABI (ctypes); the
compute path is the in-tree library ariel_b200/_lib/libariel_b200.so.
"""
from . import _abi  # noqa: F401
from ._abi import (AIR, FLUID, SOLID, AsimParams, AsimSceneDesc, AsimStats,  # noqa: F401
                   params_default, scene_dambreak)
