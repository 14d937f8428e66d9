"""B200-native (sm_100a) implementation of the MRPNN cloud-rendering path.

The compute runs in libmrpnn_b200.so (hand-written CUDA behind a C ABI,
include/mrpnn_b200.h). This package loads it with ctypes and mirrors the
reference's host interface (VolumeRender, Camera). Importing the package
loads the library and fails loudly when it has not been built.
"""
from . import _lib
from ._lib import MRError, RenderParams, load, check
from .volume import (MRPNN, PT, RPNN, Camera, Network, VolumeRender, builtin_stencil, spiral_stencil, save_bmp, tone_aces,
                     tone_gamma, tone_none, xavier_weights)

__all__ = ["VolumeRender", "Camera", "Network", "builtin_stencil", "spiral_stencil", "xavier_weights", "tone_aces", "tone_gamma",
           "tone_none", "save_bmp", "PT", "RPNN", "MRPNN", "MRError", "RenderParams", "load", "check"]

load()
