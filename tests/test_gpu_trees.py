"""GPU: the scene build's tree choices (vp_scene_options): PLOC clustering or the Karras LBVH for
the BVH32 and for the megakernel's binary tree, the BVH32 leaf size, and the SAH-optimal or greedy
collapse to BVH32.

Every choice must give the oracle's answers: transmittance within the FP64 gate of the parity
tests (2e-5 relative), ellipsoid overlap counts at points exactly.  Renders from different trees
visit the same Gaussians in another order, so they differ only in FP32 summation order: mean
|a - b| below 1e-4 of the mean image, as for the engines in test_gpu_parity.test_engines_agree.
"""
import ctypes as C
import math

import numpy as np
import pytest

import oracle as O
import volprim_b200 as vp
from volprim_b200 import _capi, scenes
from volprim_b200._capi import VP_ENGINE_MEGAKERNEL, VP_ENGINE_WARP, VP_PRECISION_ACCURATE

from test_gpu_parity import random_rays, small_scatter_workload

pytestmark = pytest.mark.gpu

COMBOS = [("ploc", "ploc", 24, "sah"), ("ploc", "ploc", 24, "greedy"), ("lbvh", "lbvh", 24, "sah"),
          ("lbvh", "lbvh", 24, "greedy"), ("ploc", "lbvh", 32, "sah"), ("lbvh", "ploc", 8, "greedy"),
          ("ploc", "ploc", 1, "sah")]


def clustered(n, seed):
    """Gaussians in a few tight clusters plus a sparse background, with a wide scale spread."""
    rng = np.random.default_rng(seed)
    centers = rng.uniform(-0.8, 0.8, (6, 3))
    which = rng.integers(0, 7, n)
    mean = np.where((which < 6)[:, None], centers[np.minimum(which, 5)] + rng.normal(0, 0.08, (n, 3)),
                    rng.uniform(-1, 1, (n, 3))).astype(np.float32)
    scale = np.exp(rng.normal(math.log(0.05), 0.6, (n, 3))).astype(np.float32)
    alb = rng.uniform(0.2, 0.9, (n, 3)).astype(np.float32)
    return vp.Gaussians(mean, scale, scenes.uniform_quaternions(rng, n),
                        np.exp(rng.normal(-1.0, 0.5, n)).astype(np.float32), alb)


@pytest.mark.parametrize("wide, binary, leaf, collapse", COMBOS)
def test_tree_choices_match_the_oracle(vp_ctx, wide, binary, leaf, collapse):
    n = 5000
    g = clustered(n, 11)
    sc = vp.Scene(vp_ctx, g, 2.0, wide_builder=wide, binary_builder=binary, leaf_max=leaf, collapse=collapse)
    info = sc.info()
    assert (info["wide_builder"], info["binary_builder"], info["leaf_max"]) == (wide, binary, leaf)
    assert info["wide_collapse"] == collapse
    assert info["leaves"] >= math.ceil(n / leaf)
    assert (info["binary_height"] > 0) == ("ploc" in (wide, binary))
    osc = O.OracleScene.from_gaussians(g, sigma_multiplier=2.0)
    rng = np.random.default_rng(12)
    o, d = random_rays(rng, 4000, radius=2.5, inside_frac=0.3)
    k = 1200
    o[:k] = g.mean[rng.choice(n, k, replace=False)]
    T64, tau64 = osc.transmittance_fp64(o, d)
    sel = tau64 < 80
    for eng in (VP_ENGINE_WARP, VP_ENGINE_MEGAKERNEL):
        T = sc.transmittance(o, d, precision=VP_PRECISION_ACCURATE, engine=eng).astype(np.float64)
        assert np.all(np.abs(T - T64)[sel] <= 2e-5 * T64[sel] + 1e-9), (eng, np.max(np.abs(T - T64)[sel]))
    pts = np.concatenate([g.mean[:2000], rng.uniform(-1, 1, (2000, 3))]).astype(np.float32)
    _, ocnt = osc.albedo_at(pts)
    for eng in (VP_ENGINE_WARP, VP_ENGINE_MEGAKERNEL):
        _, cnt = sc.albedo_at(pts, engine=eng)
        diff = np.abs(cnt.astype(np.int64) - ocnt.astype(np.int64))
        assert diff.max() <= 1 and np.mean(diff > 0) < 1e-3, (eng, diff.max())
    sc.close()


@pytest.mark.parametrize("engine", ["wavefront", "megakernel"])
def test_renders_agree_across_trees(vp_ctx, engine):
    g, cfg, env = small_scatter_workload(seed=7, n=2000, spp=16)
    cfg.engine = engine
    cam = scenes.negz_camera(3.0, 40.0)
    imgs = {}
    for key, wide, binary, collapse in (("ploc", "ploc", "ploc", "sah"), ("lbvh", "lbvh", "lbvh", "sah"),
                                        ("greedy", "ploc", "ploc", "greedy")):
        sc = vp.Scene(vp_ctx, g, 2.0, wide_builder=wide, binary_builder=binary, collapse=collapse)
        imgs[key] = vp.Renderer(cfg, sc, cam, env=env, ctx=vp_ctx).render()[..., :3]
        sc.close()
    scale = float(imgs["ploc"].mean())
    assert scale > 0.01
    assert np.abs(imgs["ploc"] - imgs["lbvh"]).mean() / scale < 1e-4
    assert np.abs(imgs["ploc"] - imgs["greedy"]).mean() / scale < 1e-4


def test_invalid_scene_options(vp_ctx):
    g = clustered(100, 3)
    for bad in ({"leaf_max": 0}, {"leaf_max": 33}):
        with pytest.raises(vp.VpError, match="leaf_max"):
            vp.Scene(vp_ctx, g, 1.0, **bad)
    with pytest.raises(ValueError):
        vp.Scene(vp_ctx, g, 1.0, collapse="optimal")
    with pytest.raises(ValueError):
        vp.Scene(vp_ctx, g, 1.0, wide_builder="sah")
    opt = _capi.vp_scene_options()
    _capi.check(_capi.lib.vp_scene_options_default(C.byref(opt)))
    opt.binary_builder = 7
    s = _capi.vp_gaussians()
    h = C.c_void_p()
    assert _capi.lib.vp_scene_create_ex(vp_ctx.handle, C.byref(s), C.c_float(1.0), C.byref(opt), C.byref(h)) == -1
    assert b"builders" in _capi.lib.vp_last_error_string()


def nested(n, seed):
    """n concentric spherical Gaussians of strictly growing scale: PLOC merges about one pair per
    pass here, so its tree is a chain of height ~n."""
    rng = np.random.default_rng(seed)
    scale = np.repeat((0.01 * 1.003 ** np.arange(n))[:, None], 3, 1).astype(np.float32)
    mean = np.zeros((n, 3), np.float32)
    return vp.Gaussians(mean, scale, scenes.uniform_quaternions(rng, n), np.full(n, 2.0 / n, np.float32),
                        np.full((n, 3), 0.5, np.float32))


def identical(n):
    q = np.tile(np.array([1.0, 0, 0, 0], np.float32), (n, 1))
    return vp.Gaussians(np.full((n, 3), 0.1, np.float32), np.full((n, 3), 0.2, np.float32), q,
                        np.full(n, 3.0 / n, np.float32), np.full((n, 3), 0.7, np.float32))


@pytest.mark.parametrize("case, wide, binary, max_height", [
    ("identical_1000", "ploc", "ploc", 16),   # buddy pairs: about log2(n) passes, a balanced tree
    ("nested_300", "ploc", "lbvh", None),     # chain of height ~300: the megakernel takes the LBVH
    ("nested_2000", "lbvh", "lbvh", 0),       # > 1024 passes: the build drops the clustering
])
def test_degenerate_layouts(vp_ctx, case, wide, binary, max_height):
    g = identical(1000) if case.startswith("identical") else nested(int(case.split("_")[1]), 5)
    sc = vp.Scene(vp_ctx, g, 1.0)
    info = sc.info()
    assert (info["wide_builder"], info["binary_builder"]) == (wide, binary), info
    if max_height is not None:
        assert info["binary_height"] <= max_height, info
    else:
        assert info["binary_height"] >= 127, info
    osc = O.OracleScene.from_gaussians(g)
    rng = np.random.default_rng(8)
    o, d = random_rays(rng, 3000, radius=3.0, inside_frac=0.3)
    o[:500] = rng.normal(0, 0.05, (500, 3))
    T64, tau64 = osc.transmittance_fp64(o, d)
    sel = tau64 < 80
    for eng in (VP_ENGINE_WARP, VP_ENGINE_MEGAKERNEL):
        T = sc.transmittance(o, d, precision=VP_PRECISION_ACCURATE, engine=eng).astype(np.float64)
        assert np.all(np.abs(T - T64)[sel] <= 2e-5 * T64[sel] + 1e-9), (eng, np.max(np.abs(T - T64)[sel]))
        pts = rng.normal(0, 0.3, (2000, 3)).astype(np.float32)
        _, cnt = sc.albedo_at(pts, engine=eng)
        _, ocnt = osc.albedo_at(pts)
        diff = np.abs(cnt.astype(np.int64) - ocnt.astype(np.int64))
        assert diff.max() <= 1 and np.mean(diff > 0) < 1e-3, (eng, diff.max())
    sc.close()
