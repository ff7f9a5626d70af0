"""Host-side mirror of the reference renderer's operator interface, over the C ABI.

Reference interface (kfernandez31/cuda-volprim):
  app::Config                        include/thesis/host/app/config.h:14-50
  app::Renderer(config, primitives, camera) + render()
                                     include/thesis/host/app/renderer.h:77-81,
                                     src/thesis/host/app/renderer.cpp:34-439
  host::params::Camera::createPerspective / createOrthographic / getDefaultCamera
                                     include/thesis/host/params/camera.h:114-150
  io::loadPrimitives (PLY semantics: log-scales, (w,x,y,z) quaternions, mass x sigma-multiplier)
                                     src/thesis/host/utils/io/ply.cpp:21-175
Differences: the image is returned in memory (H x W x 4 float32, alpha = 1) instead of written
to an EXR file, errors raise VpError instead of exiting the process, and the scene has no
65,535-Gaussian cap.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _capi
from ._capi import check, lib


def _is_cuda_tensor(x) -> bool:
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


def _sync_torch(*xs) -> None:
    """Wait for torch's current stream on the devices of the CUDA tensors among xs: the library
    runs on its own stream, so torch's pending writes to memory it reads must be complete."""
    import torch
    for dev in {x.device for x in xs if _is_cuda_tensor(x)}:
        torch.cuda.current_stream(dev).synchronize()


def _alive(ctx) -> bool:
    """Whether a wrapper's context is still open.  Scenes, environments, images and servers hold
    a pointer to their vp_context; once it is destroyed they cannot be destroyed safely, so a
    wrapper closed after its context only drops its handle (the memory goes with the process)."""
    return ctx is not None and getattr(ctx, "handle", None) is not None


def _host_f32(x, n: int, what: str) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32)).reshape(-1)
    if a.size != n:
        raise ValueError(f"{what}: expected {n} floats, got {a.size}")
    return a


class Context:
    """One CUDA device + stream (vp_context_create)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib.vp_context_create(int(device), C.byref(h)))
        self.handle = h
        self.device = device

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        check(lib.vp_context_stream(self.handle, C.byref(s)))
        return s.value or 0

    @property
    def sm_count(self) -> int:
        n = C.c_int32()
        check(lib.vp_context_sm_count(self.handle, C.byref(n)))
        return n.value

    def synchronize(self) -> None:
        check(lib.vp_context_synchronize(self.handle))

    def camera_rays(self, camera: "Camera", config: "Config", px, py, sample):
        """Camera rays of (pixel x, pixel y, sample) triples, as the renderer generates them."""
        px, py, sample = (np.ascontiguousarray(a, dtype=np.uint32).reshape(-1) for a in (px, py, sample))
        n = px.size
        o = np.empty((n, 3), np.float32)
        d = np.empty((n, 3), np.float32)
        cam, p = camera.to_c(), config.to_c()
        check(lib.vp_camera_rays(self.handle, C.byref(cam), C.byref(p), px.ctypes.data, py.ctypes.data,
                                 sample.ctypes.data, n, o.ctypes.data, d.ctypes.data, _capi.VP_MEMORY_HOST))
        return o, d

    def close(self) -> None:
        if getattr(self, "handle", None):
            lib.vp_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class Gaussians:
    """Gaussian primitive buffers in the reference's PLY semantics (ply.cpp:99-118)."""

    mean: object            # (N, 3)
    scale: object           # (N, 3) linear (or log when scale_is_log)
    quat_wxyz: object       # (N, 4) forward rotation, normalised by the library
    density: object         # (N,) total mass M per Gaussian (multiplied by sigma_multiplier)
    albedo: object = None   # (N, 3) or None
    scale_is_log: bool = False

    @property
    def count(self) -> int:
        return int(self.density.shape[0]) if hasattr(self.density, "shape") else len(self.density)


_BUILDERS = {"ploc": _capi.VP_TREE_PLOC, "lbvh": _capi.VP_TREE_LBVH}
_COLLAPSES = {"greedy": _capi.VP_COLLAPSE_GREEDY, "sah": _capi.VP_COLLAPSE_SAH}
_TAU_ORDERS = {"auto": _capi.VP_TAU_ORDER_AUTO, "lane": _capi.VP_TAU_ORDER_LANE,
               "nearest": _capi.VP_TAU_ORDER_NEAREST}


class Scene:
    """Gaussians + acceleration structure on the device (vp_scene_create_ex).

    wide_builder / binary_builder pick the binary tree of the BVH32 (warp and wavefront engines)
    and of the megakernel: "ploc" (clustering, the default) or "lbvh" (Karras radix tree);
    leaf_max is the largest BVH32 leaf (1..32); collapse cuts the BVH32 from its binary tree:
    "sah" (SAH-optimal slot assignment, the default) or "greedy" (largest area first);
    tau_order is the order transmittance queries visit a node's hit children after the nearest:
    "lane", "nearest" or "auto" (nearest when fewer than half of the Gaussians are opaque at
    their core and the BVH32 is at least 3 levels deep)."""

    def __init__(self, ctx: Context, g: Gaussians, sigma_multiplier: float = 1.0, wide_builder: str = "ploc",
                 binary_builder: str = "ploc", leaf_max: int = 24, collapse: str = "sah",
                 tau_order: str = "auto"):
        n = g.count
        if wide_builder not in _BUILDERS or binary_builder not in _BUILDERS:
            raise ValueError("builders are 'ploc' or 'lbvh'")
        if collapse not in _COLLAPSES:
            raise ValueError("collapse is 'sah' or 'greedy'")
        if tau_order not in _TAU_ORDERS:
            raise ValueError("tau_order is 'auto', 'lane' or 'nearest'")
        opt = _capi.vp_scene_options()
        check(lib.vp_scene_options_default(C.byref(opt)))
        opt.wide_builder, opt.binary_builder = _BUILDERS[wide_builder], _BUILDERS[binary_builder]
        opt.leaf_max = int(leaf_max)
        opt.wide_collapse = _COLLAPSES[collapse]
        opt.tau_order = _TAU_ORDERS[tau_order]
        self.ctx = ctx
        self._keep = []
        s = _capi.vp_gaussians()
        s.count = n
        s.scale_is_log = 1 if g.scale_is_log else 0
        if _is_cuda_tensor(g.density):
            import torch

            def dptr(t, k):
                t = t.detach().to(torch.float32).contiguous().reshape(-1)
                if t.numel() != k:
                    raise ValueError("bad tensor size")
                self._keep.append(t)
                return t.data_ptr()

            s.memory = _capi.VP_MEMORY_DEVICE
            s.mean, s.scale = dptr(g.mean, 3 * n), dptr(g.scale, 3 * n)
            s.quat_wxyz, s.density = dptr(g.quat_wxyz, 4 * n), dptr(g.density, n)
            s.albedo = dptr(g.albedo, 3 * n) if g.albedo is not None else None
            _sync_torch(*self._keep)
        else:
            arrs = [_host_f32(g.mean, 3 * n, "mean"), _host_f32(g.scale, 3 * n, "scale"),
                    _host_f32(g.quat_wxyz, 4 * n, "quat_wxyz"), _host_f32(g.density, n, "density")]
            alb = _host_f32(g.albedo, 3 * n, "albedo") if g.albedo is not None else None
            self._keep = arrs + ([alb] if alb is not None else [])
            s.memory = _capi.VP_MEMORY_HOST
            s.mean, s.scale, s.quat_wxyz, s.density = (a.ctypes.data for a in arrs)
            s.albedo = alb.ctypes.data if alb is not None else None
        h = C.c_void_p()
        check(lib.vp_scene_create_ex(ctx.handle, C.byref(s), C.c_float(sigma_multiplier), C.byref(opt), C.byref(h)))
        self.handle = h
        self._keep = []

    def info(self) -> dict:
        i = _capi.vp_scene_info()
        check(lib.vp_scene_info_get(self.handle, C.byref(i)))
        return {
            "count": i.count, "wide_nodes": i.wide_nodes, "wide_depth": i.wide_depth,
            "binary_nodes": i.binary_nodes, "albedo_all_zero": bool(i.albedo_all_zero),
            "build_ms": i.build_ms, "bounds_min": list(i.bounds_min), "bounds_max": list(i.bounds_max),
            "device_bytes": i.device_bytes, "leaves": i.leaves,
            "wide_builder": "ploc" if i.wide_builder == _capi.VP_TREE_PLOC else "lbvh",
            "binary_builder": "ploc" if i.binary_builder == _capi.VP_TREE_PLOC else "lbvh",
            "binary_height": i.binary_height, "leaf_max": i.leaf_max,
            "wide_collapse": "sah" if i.wide_collapse == _capi.VP_COLLAPSE_SAH else "greedy",
            "tau_order": "nearest" if i.tau_order == _capi.VP_TAU_ORDER_NEAREST else "lane",
        }

    def transmittance(self, origins, dirs, precision: int = _capi.VP_PRECISION_AUTO,
                      engine: int = _capi.VP_ENGINE_WARP):
        """exp(-tau) along rays over [0, inf) (vp_transmittance)."""
        if _is_cuda_tensor(origins):
            import torch
            o = origins.detach().to(torch.float32).contiguous()
            d = dirs.detach().to(torch.float32).contiguous()
            n = o.numel() // 3
            out = torch.empty(n, dtype=torch.float32, device=o.device)
            _sync_torch(o, d, out)
            check(lib.vp_transmittance(self.handle, o.data_ptr(), d.data_ptr(), n, precision, engine,
                                       out.data_ptr(), _capi.VP_MEMORY_DEVICE))
            return out
        o = np.ascontiguousarray(origins, dtype=np.float32).reshape(-1)
        d = np.ascontiguousarray(dirs, dtype=np.float32).reshape(-1)
        n = o.size // 3
        out = np.empty(n, dtype=np.float32)
        check(lib.vp_transmittance(self.handle, o.ctypes.data, d.ctypes.data, n, precision, engine,
                                   out.ctypes.data, _capi.VP_MEMORY_HOST))
        return out

    def transmittance_static(self, origins, dirs, precision: int = _capi.VP_PRECISION_AUTO):
        """vp_transmittance_static: the transmittance query with no device allocation (its scratch
        is a static device array for at most 65536 rays per call; calls must not overlap)."""
        if _is_cuda_tensor(origins):
            import torch
            o = origins.detach().to(torch.float32).contiguous()
            d = dirs.detach().to(torch.float32).contiguous()
            n = o.numel() // 3
            out = torch.empty(n, dtype=torch.float32, device=o.device)
            _sync_torch(o, d, out)
            check(lib.vp_transmittance_static(self.handle, o.data_ptr(), d.data_ptr(), n, precision, out.data_ptr(),
                                              _capi.VP_MEMORY_DEVICE))
            return out
        o = np.ascontiguousarray(origins, dtype=np.float32).reshape(-1)
        d = np.ascontiguousarray(dirs, dtype=np.float32).reshape(-1)
        n = o.size // 3
        out = np.empty(n, dtype=np.float32)
        check(lib.vp_transmittance_static(self.handle, o.ctypes.data, d.ctypes.data, n, precision, out.ctypes.data,
                                          _capi.VP_MEMORY_HOST))
        return out

    def set_emission(self, rgb):
        """RGB emission per unit optical depth, (count, 3) in the order the scene was built from
        (vp_scene_set_emission); a host array or a CUDA tensor."""
        n = self.info()["count"]
        if _is_cuda_tensor(rgb):
            import torch
            t = rgb.detach().to(torch.float32).contiguous().reshape(-1)
            if t.numel() != 3 * n:
                raise ValueError(f"emission: expected {3 * n} floats, got {t.numel()}")
            _sync_torch(t)
            check(lib.vp_scene_set_emission(self.handle, t.data_ptr(), _capi.VP_MEMORY_DEVICE))
            return
        a = _host_f32(rgb, 3 * n, "emission")
        check(lib.vp_scene_set_emission(self.handle, a.ctypes.data, _capi.VP_MEMORY_HOST))

    def albedo_at(self, points, precision: int = _capi.VP_PRECISION_AUTO, engine: int = _capi.VP_ENGINE_WARP):
        """(albedo rgb (n, 3), overlap count (n,)) at points (vp_albedo_at)."""
        p = np.ascontiguousarray(points, dtype=np.float32).reshape(-1)
        n = p.size // 3
        rgb = np.empty((n, 3), dtype=np.float32)
        cnt = np.empty(n, dtype=np.uint32)
        check(lib.vp_albedo_at(self.handle, p.ctypes.data, n, precision, engine, rgb.ctypes.data, cnt.ctypes.data,
                               _capi.VP_MEMORY_HOST))
        return rgb, cnt

    def close(self):
        if getattr(self, "handle", None):
            if _alive(self.ctx):
                lib.vp_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Environment:
    """Lat-long HDR environment + importance-sampling tables (vp_env_create)."""

    def __init__(self, ctx: Context, rgb=None, constant=None):
        h = C.c_void_p()
        self.ctx = ctx
        if constant is not None:
            r, g, b = (float(v) for v in constant)
            check(lib.vp_env_create_constant(ctx.handle, r, g, b, C.byref(h)))
        else:
            if _is_cuda_tensor(rgb):
                import torch
                t = rgb.detach().to(torch.float32).contiguous()
                hgt, wid, ch = t.shape
                _sync_torch(t)
                check(lib.vp_env_create(ctx.handle, t.data_ptr(), wid, hgt, ch, _capi.VP_MEMORY_DEVICE,
                                        C.byref(h)))
            else:
                a = np.ascontiguousarray(rgb, dtype=np.float32)
                hgt, wid, ch = a.shape
                check(lib.vp_env_create(ctx.handle, a.ctypes.data, wid, hgt, ch, _capi.VP_MEMORY_HOST,
                                        C.byref(h)))
        self.handle = h

    @property
    def build_ms(self) -> float:
        v = C.c_double()
        check(lib.vp_env_build_ms(self.handle, C.byref(v)))
        return v.value

    def tables(self) -> dict:
        """The device-built sampling tables (vp_env_read_tables): per texel the alias probability,
        alias texel and joint weight (H x W), per row the marginal alias probability and row, and
        the total weight."""
        w, h, tot = C.c_uint32(), C.c_uint32(), C.c_float()
        check(lib.vp_env_read_tables(self.handle, C.byref(w), C.byref(h), None, None, None, None, None, None))
        W, H = w.value, h.value
        t = {"cond_prob": np.empty((H, W), np.float32), "cond_alias": np.empty((H, W), np.uint32),
             "marg_prob": np.empty(H, np.float32), "marg_alias": np.empty(H, np.uint32),
             "joint": np.empty((H, W), np.float32)}
        check(lib.vp_env_read_tables(self.handle, None, None, *(t[k].ctypes.data for k in
                                     ("cond_prob", "cond_alias", "marg_prob", "marg_alias", "joint")), C.byref(tot)))
        t["total"] = tot.value
        return t

    def close(self):
        if getattr(self, "handle", None):
            if _alive(self.ctx):
                lib.vp_env_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class Camera:
    """host::params::Camera (include/thesis/host/params/camera.h:18-166)."""

    eye: tuple = (0.0, 0.0, -1.0)
    lookat: tuple = (0.0, 0.0, 0.0)
    up: tuple = (0.0, 1.0, 0.0)
    vfov_deg: float = 90.0
    ortho_height: float = 2.0
    orthographic: bool = False

    @staticmethod
    def perspective(origin, target, up, vertical_fov_deg: float) -> "Camera":
        return Camera(tuple(origin), tuple(target), tuple(up), float(vertical_fov_deg), 2.0, False)

    @staticmethod
    def orthographic_camera(origin, target, up, ortho_height: float) -> "Camera":
        return Camera(tuple(origin), tuple(target), tuple(up), 90.0, float(ortho_height), True)

    @staticmethod
    def default() -> "Camera":  # getDefaultCamera (include/thesis/host/params/camera.h:117-121)
        return Camera()

    def to_c(self) -> _capi.vp_camera:
        c = _capi.vp_camera()
        c.eye[:] = [float(v) for v in self.eye]
        c.lookat[:] = [float(v) for v in self.lookat]
        c.up[:] = [float(v) for v in self.up]
        c.vfov_deg = self.vfov_deg
        c.ortho_height = self.ortho_height
        c.orthographic = 1 if self.orthographic else 0
        return c


@dataclass
class Config:
    """Render controls of app::Config (config.h:14-50) plus this library's engine choices."""

    num_samples_per_pixel: int = 1
    image_width: int = 1000
    image_height: int = 750
    seed: int = 42
    max_bounces: int = 128
    rr_depth: int = 12
    rr_max_survival: float = 0.99
    firefly_clamp_luminance: float = 0.0
    pixel_filter_stddev: float = 0.0
    hg_g: float = 0.85
    use_ris: bool = False
    ris_num_candidates: int = 6
    measure_caps: bool = False  # device counters (VP_MEASURE_COUNTERS)
    time_stages: bool = False   # CUDA-event time of the wavefront stages (VP_MEASURE_STAGES)
    nee: str = "mis"            # "mis" | "phase" | "ris" | "none"  (use_ris=True selects "ris")
    engine: str = "wavefront"   # "wavefront" | "warp" | "megakernel"
    precision: str = "auto"     # "auto" | "fast" | "accurate"
    batch_spp: int = 16         # BATCH_SIZE (renderer.cpp:32)
    # adaptive sampling (ADAPTIVE_THRESHOLD / ADAPTIVE_MIN_SAMPLES, constants.cuh:196-211): a pixel
    # with at least adaptive_min_samples samples whose largest per-channel std-dev / mean is below
    # adaptive_threshold takes no more batches; 0 = off (the reference's default)
    adaptive_threshold: float = 0.0
    adaptive_min_samples: int = 32

    def to_c(self) -> _capi.vp_render_params:
        p = _capi.vp_render_params()
        check(lib.vp_render_params_default(C.byref(p)))
        p.width, p.height = self.image_width, self.image_height
        p.spp, p.seed = self.num_samples_per_pixel, self.seed
        p.max_bounces, p.rr_depth = self.max_bounces, self.rr_depth
        p.rr_max_survival, p.hg_g = self.rr_max_survival, self.hg_g
        p.firefly_clamp, p.pixel_filter_stddev = self.firefly_clamp_luminance, self.pixel_filter_stddev
        nee = "ris" if self.use_ris else self.nee
        p.nee_mode = {"mis": 0, "phase": 1, "ris": 2, "none": 3}[nee]
        p.ris_candidates = self.ris_num_candidates
        p.batch_spp = self.batch_spp
        p.engine = {"warp": 0, "megakernel": 1, "wavefront": 2}[self.engine]
        p.precision = {"auto": 0, "fast": 1, "accurate": 2}[self.precision]
        p.measure = ((_capi.VP_MEASURE_COUNTERS if self.measure_caps else 0)
                     | (_capi.VP_MEASURE_STAGES if self.time_stages else 0))
        p.adaptive_threshold, p.adaptive_min_samples = self.adaptive_threshold, self.adaptive_min_samples
        return p


class Renderer:
    """app::Renderer(config, primitives, camera) + render() over the C ABI.

    `primitives` is a Gaussians record or an already-built Scene; `env` is an Environment, an
    (H, W, C) array, or None for the constant white environment.
    """

    def __init__(self, config: Config, primitives, camera: Optional[Camera] = None, env=None,
                 sigma_multiplier: float = 1.0, ctx: Optional[Context] = None):
        self.config = config
        self.ctx = ctx or (primitives.ctx if isinstance(primitives, Scene) else Context(0))
        self.scene = primitives if isinstance(primitives, Scene) else Scene(self.ctx, primitives, sigma_multiplier)
        if isinstance(env, Environment):
            self.env = env
        elif env is None:
            self.env = Environment(self.ctx, constant=(1.0, 1.0, 1.0))
        else:
            self.env = Environment(self.ctx, rgb=env)
        self.camera = camera or Camera.default()
        self.last_stats: dict = {}

    def render(self, out=None):
        """Whole render; returns an (H, W, 4) float32 array (or fills the torch CUDA tensor `out`)."""
        p = self.config.to_c()
        cam = self.camera.to_c()
        st = _capi.vp_render_stats()
        if out is not None and _is_cuda_tensor(out):
            _sync_torch(out)
            check(lib.vp_render(self.scene.handle, self.env.handle, C.byref(cam), C.byref(p), out.data_ptr(),
                                _capi.VP_MEMORY_DEVICE, C.byref(st)))
            self.last_stats = st.as_dict()
            return out
        img = np.empty((p.height, p.width, 4), dtype=np.float32)
        check(lib.vp_render(self.scene.handle, self.env.handle, C.byref(cam), C.byref(p), img.ctypes.data,
                            _capi.VP_MEMORY_HOST, C.byref(st)))
        self.last_stats = st.as_dict()
        return img


class ProgressiveImage:
    """Welford accumulation image (vp_image_*), for rendering sample ranges incrementally."""

    def __init__(self, ctx: Context, width: int, height: int):
        h = C.c_void_p()
        check(lib.vp_image_create(ctx.handle, width, height, C.byref(h)))
        self.handle, self.ctx, self.width, self.height = h, ctx, width, height

    def clear(self):
        check(lib.vp_image_clear(self.handle))

    def accumulate(self, scene: Scene, env: Environment, camera: Camera, config: Config,
                   spp_offset: int, spp_count: int) -> dict:
        p = config.to_c()
        cam = camera.to_c()
        st = _capi.vp_render_stats()
        check(lib.vp_render_accumulate(scene.handle, env.handle, C.byref(cam), C.byref(p), self.handle,
                                       spp_offset, spp_count, C.byref(st)))
        return st.as_dict()

    def read(self) -> np.ndarray:
        img = np.empty((self.height, self.width, 4), dtype=np.float32)
        check(lib.vp_image_read(self.handle, img.ctypes.data, _capi.VP_MEMORY_HOST))
        return img

    def read_welford(self, m2: bool = True):
        """(M2 (H, W, 3) float32 or None, sample counts (H, W) uint32).  M2 exists only while every
        batch since the last clear ran with adaptive sampling on."""
        q = np.empty((self.height, self.width, 4), dtype=np.float32) if m2 else None
        n = np.empty((self.height, self.width), dtype=np.uint32)
        check(lib.vp_image_read_welford(self.handle, q.ctypes.data if m2 else None, n.ctypes.data,
                                        _capi.VP_MEMORY_HOST))
        return (q[..., :3] if m2 else None), n

    def close(self):
        if getattr(self, "handle", None):
            if _alive(self.ctx):
                lib.vp_image_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
