"""Absorption-plus-emission image and its adjoint over the C ABI (vp_render_emission,
vp_render_emission_backward).  The reference renderer has neither; the image model is the one
include/volprim_b200.h states:

    L = (1 - T) C / S + T env(d),   S = sum tau_i,  C = sum tau_i e_i,  T = exp(-S)

per jittered camera ray, averaged over spp (box filter).  The model has no occlusion between
Gaussians: a Gaussian behind an opaque one still contributes its tau-weighted share of the colour;
only the background is attenuated (by the exact transmittance T).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import check, lib
from .api import Camera, Config, Environment, Scene, _is_cuda_tensor, _sync_torch


def render_emission(scene: Scene, env: Environment, camera: Camera, config: Config, out=None, stats: dict | None = None):
    """(H, W, 4) float32 image; into `out` (a CUDA tensor) when given, else a new host array.
    `stats`, when given, receives the call's vp_render_stats."""
    p, cam = config.to_c(), camera.to_c()
    st = _capi.vp_render_stats()
    if out is not None and _is_cuda_tensor(out):
        if not out.is_contiguous() or out.numel() != 4 * config.image_width * config.image_height:
            raise ValueError("out must be a contiguous (H, W, 4) float32 CUDA tensor")
        _sync_torch(out)
        check(lib.vp_render_emission(scene.handle, env.handle, C.byref(cam), C.byref(p), out.data_ptr(),
                                     _capi.VP_MEMORY_DEVICE, C.byref(st)))
        if stats is not None:
            stats.update(st.as_dict())
        return out
    img = np.empty((config.image_height, config.image_width, 4), dtype=np.float32)
    check(lib.vp_render_emission(scene.handle, env.handle, C.byref(cam), C.byref(p), img.ctypes.data,
                                 _capi.VP_MEMORY_HOST, C.byref(st)))
    if stats is not None:
        stats.update(st.as_dict())
    return img


def render_emission_backward(scene: Scene, env: Environment, camera: Camera, config: Config, dloss_drgba,
                             grads: dict) -> dict:
    """Adds dLoss/dparam into grads["mean"], ["scale"], ["quat_wxyz"], ["density"] and (optional)
    ["emission"]: all host float32 arrays or all CUDA float32 tensors of the scene's sizes, in
    the caller's order.  dloss_drgba: (H, W, 4) (alpha ignored).  Returns the call's stats."""
    p, cam = config.to_c(), camera.to_c()
    st = _capi.vp_render_stats()
    g = _capi.vp_gaussian_grads()
    keys = ("mean", "scale", "quat_wxyz", "density", "emission")
    dev = _is_cuda_tensor(grads["mean"])
    for k in keys:
        a = grads.get(k)
        if a is None:
            if k != "emission":
                raise ValueError(f"grads[{k!r}] is required")
            setattr(g, k, None)
            continue
        if dev:
            if not (_is_cuda_tensor(a) and a.is_contiguous() and str(a.dtype) == "torch.float32"):
                raise ValueError("gradient arrays must all be contiguous float32 CUDA tensors")
            setattr(g, k, a.data_ptr())
        else:
            if not (isinstance(a, np.ndarray) and a.dtype == np.float32 and a.flags.c_contiguous):
                raise ValueError("gradient arrays must all be contiguous float32 numpy arrays")
            setattr(g, k, a.ctypes.data)
    g.memory = _capi.VP_MEMORY_DEVICE if dev else _capi.VP_MEMORY_HOST
    if _is_cuda_tensor(dloss_drgba):
        import torch
        dl = dloss_drgba.detach().to(torch.float32).contiguous()
        _sync_torch(dl, *[grads[k] for k in keys if grads.get(k) is not None])
        check(lib.vp_render_emission_backward(scene.handle, env.handle, C.byref(cam), C.byref(p), dl.data_ptr(),
                                              _capi.VP_MEMORY_DEVICE, C.byref(g), C.byref(st)))
    else:
        dl = np.ascontiguousarray(dloss_drgba, dtype=np.float32)
        if dev:
            _sync_torch(*[grads[k] for k in keys if grads.get(k) is not None])
        check(lib.vp_render_emission_backward(scene.handle, env.handle, C.byref(cam), C.byref(p), dl.ctypes.data,
                                              _capi.VP_MEMORY_HOST, C.byref(g), C.byref(st)))
    return st.as_dict()
