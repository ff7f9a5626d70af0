"""volprim_b200: B200-native per-ray hot path of a Gaussian kernel-mixture volumetric path tracer
(analog decomposition tracking, NEE/MIS, environment importance sampling) behind a C ABI
(include/volprim_b200.h), with a host-side mirror of the reference renderer's interface."""
from ._capi import (VP_ENGINE_MEGAKERNEL, VP_ENGINE_WARP, VP_NEE_MIS, VP_NEE_NONE, VP_NEE_PHASE,
                    VP_NEE_RIS, VP_PRECISION_ACCURATE, VP_PRECISION_AUTO, VP_PRECISION_FAST, VpError,
                    LIB_PATH)
from .api import Camera, Config, Context, Environment, Gaussians, ProgressiveImage, Renderer, Scene

__all__ = [
    "Camera", "Config", "Context", "Environment", "Gaussians", "ProgressiveImage", "Renderer", "Scene",
    "VpError", "LIB_PATH", "VP_ENGINE_WARP", "VP_ENGINE_MEGAKERNEL", "VP_NEE_MIS", "VP_NEE_PHASE",
    "VP_NEE_RIS", "VP_NEE_NONE", "VP_PRECISION_AUTO", "VP_PRECISION_FAST", "VP_PRECISION_ACCURATE",
]
