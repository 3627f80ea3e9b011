"""B200-native textured 2DGS rasterization (forward + backward).

Drop-in for the hot path of Camak2441/textured_gaussians: the renderer API in
:mod:`textured_gaussians_b200.rendering` and the op surface in
:mod:`textured_gaussians_b200.cuda`, all backed by hand-written sm_100a
kernels in ``libtg2dgs.so`` (C ABI: include/tg2dgs.h).
"""
from .rendering import rasterization_2dgs, rasterization_textured_gaussians

__all__ = ["rasterization_2dgs", "rasterization_textured_gaussians"]
__version__ = "0.1.0"
