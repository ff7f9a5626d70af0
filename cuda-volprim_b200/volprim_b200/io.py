"""Asset IO over the C ABI: Gaussian PLY files (vp_ply_load / vp_ply_save), Radiance RGBE
environment maps (vp_hdr_load) and OpenEXR images (vp_exr_save), with the reference's semantics
(src/thesis/host/utils/io/ply.cpp, hdr.cpp, exr.cpp)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _capi
from ._capi import check, lib
from .api import Gaussians


def load_ply(path, albedo_override=None) -> Gaussians:
    """The file's Gaussians as host arrays (log-scales: scale_is_log=True); density is the total
    mass before the sigma-multiplier.  albedo_override (3 floats) replaces the file's albedo when
    all three are >= 0."""
    g = _capi.vp_host_gaussians()
    ov = None
    if albedo_override is not None:
        ov = np.ascontiguousarray(albedo_override, np.float32).reshape(3)
    check(lib.vp_ply_load(os.fsencode(str(path)), ov.ctypes.data if ov is not None else None, C.byref(g)))
    try:
        n = g.count

        def arr(ptr, k):
            return np.ctypeslib.as_array(ptr, shape=(n * k,)).copy().reshape(n, k) if n else np.zeros((0, k), np.float32)

        out = Gaussians(arr(g.mean, 3), arr(g.log_scale, 3), arr(g.quat_wxyz, 4), arr(g.density, 1).reshape(n),
                        arr(g.albedo, 3), scale_is_log=True)
    finally:
        lib.vp_host_gaussians_free(C.byref(g))
    return out


def save_ply(path, g: Gaussians) -> None:
    """Writes the 14 properties (binary little-endian floats); g's scales must be logs."""
    if not g.scale_is_log:
        raise ValueError("save_ply stores log-scales: pass Gaussians(scale_is_log=True)")
    n = g.count
    arrs = [np.ascontiguousarray(a, np.float32).reshape(-1) for a in (g.mean, g.scale, g.quat_wxyz, g.density)]
    alb = np.ascontiguousarray(g.albedo if g.albedo is not None else np.zeros((n, 3)), np.float32).reshape(-1)
    h = _capi.vp_host_gaussians()
    h.count = n
    fp = C.POINTER(C.c_float)
    h.mean, h.log_scale, h.quat_wxyz, h.density = (a.ctypes.data_as(fp) for a in arrs)
    h.albedo = alb.ctypes.data_as(fp)
    check(lib.vp_ply_save(os.fsencode(str(path)), C.byref(h)))


def load_hdr(path) -> np.ndarray:
    """(H, W, 3) float32 radiance of a Radiance RGBE file (row 0 = the first scanline)."""
    p = C.POINTER(C.c_float)()
    w, h = C.c_uint32(), C.c_uint32()
    check(lib.vp_hdr_load(os.fsencode(str(path)), C.byref(p), C.byref(w), C.byref(h)))
    try:
        return np.ctypeslib.as_array(p, shape=(h.value * w.value * 3,)).copy().reshape(h.value, w.value, 3)
    finally:
        lib.vp_host_free(p)


def save_exr(path, rgba, flip_vertical: bool = False) -> None:
    """Writes an (H, W, 4) (or (H, W, 3)) float image as an OpenEXR file (FLOAT B, G, R)."""
    a = np.asarray(rgba, np.float32)
    if a.ndim != 3 or a.shape[2] not in (3, 4):
        raise ValueError("expected an (H, W, 3|4) image")
    if a.shape[2] == 3:
        a = np.concatenate([a, np.ones(a.shape[:2] + (1,), np.float32)], axis=2)
    a = np.ascontiguousarray(a)
    check(lib.vp_exr_save(os.fsencode(str(path)), a.ctypes.data, a.shape[1], a.shape[0], 1 if flip_vertical else 0))
