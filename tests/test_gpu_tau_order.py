"""GPU: the order in which transmittance queries visit a node's hit children (vp_tau_order).

AUTO picks NEAREST for scenes of many overlapping, individually translucent Gaussians (the stress
generator's kind) and LANE for scenes whose Gaussians are opaque at their core (the showcase
generator's kind) or whose BVH32 is too shallow to order (the 256-Gaussian absorption case).
The order changes only the summation order of the optical depth and how soon a ray stops at
MAX_OPTICAL_DEPTH, so:
  ACCURATE (float-pair sums): |T_lane - T_nearest| <= 1e-6 T + 1e-12;
  FAST (FP32 sums of up to a few hundred chords: relative tau error up to ~1e-5, so up to ~1e-4
  relative in T for tau ~ 10): <= 1e-3 T + 1e-9;
  a wavefront render (transmittance draws no random numbers, so the paths are the same): mean
  |difference| / mean < 1e-5 and >= 99% of pixels within 1e-4 relative + 1e-6.
"""
import numpy as np
import pytest

import volprim_b200 as vp
from volprim_b200 import scenes
from volprim_b200._capi import VP_PRECISION_ACCURATE, VP_PRECISION_FAST

pytestmark = pytest.mark.gpu


def rays(rng, g, n):
    k = n // 2
    o = np.concatenate([g.mean[rng.choice(len(g.density), k, replace=k > len(g.density))],
                        3.0 * rng.normal(size=(n - k, 3))]).astype(np.float64)
    o[k:] *= 3.0 / np.linalg.norm(o[k:], axis=1, keepdims=True)
    d = rng.normal(size=(n, 3))
    d[k:] = rng.uniform(-0.6, 0.6, (n - k, 3)) - o[k:]
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return o.astype(np.float32), d.astype(np.float32)


WORLDS = {
    "stress": (lambda: scenes.stress_gaussians(100_000, 3), 1.0, "nearest"),
    "showcase": (lambda: scenes.showcase_gaussians(100_000, 3), 7.5, "lane"),
    "absorption": (lambda: scenes.absorption_gaussians(256, 0), 1.0, "lane"),
}


@pytest.mark.parametrize("name", sorted(WORLDS))
def test_auto_choice_and_orders_agree(vp_ctx, name):
    make, sigma, expect = WORLDS[name]
    g = make()
    auto = vp.Scene(vp_ctx, g, sigma)
    assert auto.info()["tau_order"] == expect
    auto.close()
    sc = {k: vp.Scene(vp_ctx, g, sigma, tau_order=k) for k in ("lane", "nearest")}
    assert sc["lane"].info()["tau_order"] == "lane" and sc["nearest"].info()["tau_order"] == "nearest"
    o, d = rays(np.random.default_rng(11), g, 20000)
    for prec, rel, abs_ in ((VP_PRECISION_ACCURATE, 1e-6, 1e-12), (VP_PRECISION_FAST, 1e-3, 1e-9)):
        ta = sc["lane"].transmittance(o, d, precision=prec).astype(np.float64)
        tb = sc["nearest"].transmittance(o, d, precision=prec).astype(np.float64)
        assert (ta < 0.99).sum() > 1000  # the rays cross Gaussians (in the stress scene nearly all become opaque)
        bad = np.abs(ta - tb) > rel * np.maximum(ta, tb) + abs_
        assert not bad.any(), (prec, int(bad.sum()), float(np.max(np.abs(ta - tb))))
    for s in sc.values():
        s.close()


def test_orders_render_the_same_image(vp_ctx):
    g = scenes.stress_gaussians(100_000, 4)
    env = scenes.procedural_env(256, 128, sun_radiance=200.0, sun_radius_deg=3.0)
    cfg = vp.Config(num_samples_per_pixel=16, image_width=64, image_height=64, seed=3, hg_g=0.0,
                    max_bounces=32, rr_depth=8, nee="mis", engine="wavefront")
    cam = scenes.negz_camera()
    imgs = {}
    for k in ("lane", "nearest"):
        sc = vp.Scene(vp_ctx, g, 1.0, tau_order=k)
        imgs[k] = vp.Renderer(cfg, sc, cam, env=env, ctx=vp_ctx).render()[..., :3].astype(np.float64)
        sc.close()
    a, b = imgs["lane"], imgs["nearest"]
    assert a.mean() > 1e-3
    assert np.abs(a - b).mean() / a.mean() < 1e-5
    assert np.mean(np.abs(a - b) <= 1e-4 * np.abs(a) + 1e-6) >= 0.99


def test_invalid_order_raises(vp_ctx):
    g = scenes.absorption_gaussians(16, 0)
    with pytest.raises(ValueError):
        vp.Scene(vp_ctx, g, tau_order="sorted")
