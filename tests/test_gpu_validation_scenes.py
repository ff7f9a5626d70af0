"""GPU: the reference test runner's geometric validation scenes (test/scenes/
geometric_validation.cpp; tests/validation_scenes.py) as regression fixtures, every one
through every engine.

Per scene:
- transmittance of the runner camera's rays (eye (0, 0, -1), vfov 90) and of rays from random
  origins in and around the scene, ACCURATE, warp and megakernel engines, against the oracle's
  FP64 closed form: |T - T64| <= 2e-5 T64 + 1e-9 where tau < 80 (the parity gate);
- overlap counts and blended albedo at the Gaussians' centres and random points against the
  oracle (counts exact up to points on a 3-sigma boundary);
- a scattering render with the runner's render defaults (HG g = 0.85, MIS NEE, roulette from depth
  12, max depth 128) under the procedural environment, wavefront and warp engines, against the
  keyed oracle: the same estimator with the same random numbers, so pixels agree to FP32 noise
  except where an FP32 rounding sends a path another way (mean |difference| / mean below 1e-3 and
  at least 90 % of the pixels within 1e-3).
The empty scene (the reference's IAS over zero instances) gives T = 1 and no overlaps and renders
the environment.  Every scene renders with device status 0 (no error word from any kernel).
"""
import numpy as np
import pytest

import oracle as O
import volprim_b200 as vp
from volprim_b200 import scenes
import validation_scenes as VS
from volprim_b200._capi import VP_ENGINE_MEGAKERNEL, VP_ENGINE_WARP, VP_PRECISION_ACCURATE

pytestmark = pytest.mark.gpu

SCENES = VS.validation_scenes()
W, H, SPP = 24, 18, 8


@pytest.fixture(scope="module")
def env_pair(vp_ctx):
    rgb = scenes.procedural_env(64, 32, sun_radiance=50.0, sun_radius_deg=8.0)
    return vp.Environment(vp_ctx, rgb=rgb), O.OracleEnv(rgb)


def probe_rays(g, rng, cam16):
    """Camera rays of every pixel of a W x H image plus rays from random origins near the scene
    (half of them inside its Gaussians' 3-sigma boxes) in random directions."""
    px, py = np.meshgrid(np.arange(W), np.arange(H))
    o_cam, d_cam = O.camera_rays(cam16, W, 1, 42, px.ravel(), py.ravel(), np.zeros(W * H))
    n = 800
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    if g.count:
        k = rng.integers(0, g.count, n)
        o = g.mean[k] + rng.normal(size=(n, 3)) * 1.5 * g.scale[k]
    else:
        o = rng.uniform(-2, 2, (n, 3))
    return (np.concatenate([o_cam, o.astype(np.float32)]), np.concatenate([d_cam, d.astype(np.float32)]))


@pytest.mark.parametrize("sc", SCENES, ids=[s.name for s in SCENES])
def test_validation_scene_queries(vp_ctx, sc):
    g = sc.gaussians
    scene = vp.Scene(vp_ctx, g, 1.0)
    osc = O.OracleScene.from_gaussians(g, sigma_multiplier=1.0)
    rng = np.random.default_rng(17)
    cam16 = O.camera16(VS.runner_camera(), W, H)
    o, d = probe_rays(g, rng, cam16)
    T64, tau64 = osc.transmittance_fp64(o, d)
    sel = tau64 < 80
    for eng in (VP_ENGINE_WARP, VP_ENGINE_MEGAKERNEL):
        T = scene.transmittance(o, d, precision=VP_PRECISION_ACCURATE, engine=eng).astype(np.float64)
        err = np.abs(T - T64)
        assert np.all(err[sel] <= 2e-5 * T64[sel] + 1e-9), (eng, np.max(err[sel] / np.maximum(T64[sel], 1e-30)))
        assert np.all(T[tau64 > 90] == 0.0), eng
    if g.count == 0:
        assert np.all(T64 == 1.0)
    pts = np.concatenate([g.mean, o[W * H:] + 0.3 * d[W * H:]]).astype(np.float32)
    orgb, ocnt = osc.albedo_at(pts)
    for eng in (VP_ENGINE_WARP, VP_ENGINE_MEGAKERNEL):
        rgb, cnt = scene.albedo_at(pts, engine=eng)
        diff = np.abs(cnt.astype(np.int64) - ocnt.astype(np.int64))
        assert diff.max(initial=0) <= 1 and np.mean(diff > 0) < 5e-3, (eng, diff.max())
        same = diff == 0
        np.testing.assert_allclose(rgb[same], orgb[same], atol=1e-5)
    scene.close()


@pytest.mark.parametrize("engine", ["wavefront", "warp"])
@pytest.mark.parametrize("sc", SCENES, ids=[s.name for s in SCENES])
def test_validation_scene_render(vp_ctx, env_pair, sc, engine):
    env, oenv = env_pair
    cfg = vp.Config(num_samples_per_pixel=SPP, image_width=W, image_height=H, seed=42, engine=engine)
    cam = VS.runner_camera()
    r = vp.Renderer(cfg, vp.Scene(vp_ctx, sc.gaussians, 1.0), cam, env=env, ctx=vp_ctx)
    img = r.render()[..., :3]
    assert r.last_stats["device_status"] == 0
    osc = O.OracleScene.from_gaussians(sc.gaussians, sigma_multiplier=1.0)
    ref, _ = O.render(osc, oenv, O.camera16(cam, W, H), cfg, rng_mode="keyed")
    scale = max(float(ref.mean()), 1e-6)
    rel = np.abs(img - ref) / np.maximum(np.abs(ref), 0.05 * scale)
    frac = float(np.mean(rel < 1e-3))
    mean_rel = float(np.abs(img - ref).mean() / scale)
    assert frac >= 0.9 and mean_rel < 1e-3, (sc.name, engine, frac, mean_rel)
    r.scene.close()
