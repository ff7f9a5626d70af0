"""GPU: adaptive sampling (device/core/constants.cuh:196-211; device/entry/raygen.cuh:52-67 and
:210-242) in every render engine.

- M2, the Welford sum of squared deviations the image keeps, equals the FP64 sum over the same
  paths' radiances, rendered one sample at a time (1e-4 relative: FP32 Welford order).
- The skip decision is the oracle's test on the image's own state, exactly: a pixel whose
  (mean, M2, count) before a batch passes it keeps that state bit for bit, every other pixel
  takes the whole batch; the skipped paths are counted.
- Against the oracle's progressive render (CPU, FP32, keyed): the same pixels stop, up to the
  few whose statistic sits within the FP32 difference of the two renders of the threshold.
- Errors: an invalid threshold, an adaptive batch on an image whose earlier batches kept no M2,
  a served request with adaptive sampling.
"""
import dataclasses

import numpy as np
import pytest

import oracle as O
import volprim_b200 as vp
from volprim_b200 import scenes

from test_gpu_parity import small_scatter_workload

pytestmark = pytest.mark.gpu

ENGINES = ["wavefront", "warp", "megakernel"]
NEVER = 1 << 30  # a minimum sample count no pixel reaches: M2 is kept, nothing is skipped


def workload(vp_ctx, engine, spp, res=16, seed=5):
    g, cfg, envimg = small_scatter_workload(seed=seed, n=300, res=res, spp=spp)
    cfg.engine = engine
    cfg.batch_spp = 8
    scene = vp.Scene(vp_ctx, g, 2.0)
    env = vp.Environment(vp_ctx, rgb=envimg)
    return g, cfg, envimg, scene, env, scenes.negz_camera(3.0, 40.0)


def state_of(img):
    m2, cnt = img.read_welford()
    return img.read()[..., :3].copy(), m2.copy(), cnt.copy()


def threshold_for(vp_ctx, scene, env, cam, cfg, frac, after=16):
    """A threshold that about `frac` of the pixels pass after `after` samples (the statistic's
    quantile on a probe render of the same paths)."""
    probe = vp.ProgressiveImage(vp_ctx, cfg.image_width, cfg.image_height)
    probe.accumulate(scene, env, cam, dataclasses.replace(cfg, adaptive_threshold=1.0, adaptive_min_samples=NEVER),
                     0, after)
    mean, m2, cnt = state_of(probe)
    probe.close()
    err = np.max(np.sqrt(m2 / (cnt[..., None] - 1.0)) / np.maximum(mean, 1e-6), axis=-1)
    return float(np.quantile(err, frac))


@pytest.mark.parametrize("engine", ENGINES)
def test_m2_matches_per_sample_radiance(vp_ctx, engine):
    spp = 24
    g, cfg, _, scene, env, cam = workload(vp_ctx, engine, spp)
    W = H = cfg.image_width
    per = np.empty((spp, H, W, 3), np.float64)
    one = vp.ProgressiveImage(vp_ctx, W, H)
    for s in range(spp):  # a first sample's mean is that sample's radiance
        one.clear()
        one.accumulate(scene, env, cam, cfg, s, 1)
        per[s] = one.read()[..., :3]
    cfg.adaptive_threshold, cfg.adaptive_min_samples = 1.0, NEVER
    img = vp.ProgressiveImage(vp_ctx, W, H)
    st = img.accumulate(scene, env, cam, cfg, 0, spp)
    mean, m2, cnt = state_of(img)
    assert st["paths_skipped"] == 0 and st["paths"] == W * H * spp and st["device_status"] == 0
    assert np.all(cnt == spp)
    scale = float(per.mean())
    assert scale > 0.01
    np.testing.assert_allclose(mean, per.mean(0), rtol=1e-4, atol=1e-6 * scale)
    want = ((per - per.mean(0)) ** 2).sum(0)
    np.testing.assert_allclose(m2, want, rtol=1e-4, atol=1e-5 * scale * scale)
    assert want.max() > 0.0
    one.close()
    img.close()
    scene.close()


@pytest.mark.parametrize("engine", ENGINES)
def test_skips_follow_the_test_on_the_image_state(vp_ctx, engine):
    spp, nmin = 64, 16
    g, cfg, _, scene, env, cam = workload(vp_ctx, engine, spp, res=24)
    W = H = cfg.image_width
    thr = threshold_for(vp_ctx, scene, env, cam, cfg, 0.5)
    cfg.adaptive_threshold, cfg.adaptive_min_samples = thr, nmin
    img = vp.ProgressiveImage(vp_ctx, W, H)
    before = state_of(img)
    total_skipped = 0
    for b0 in range(0, spp, 8):
        st = img.accumulate(scene, env, cam, cfg, b0, 8)
        after = state_of(img)
        conv = O.adaptive_converged(before[0], before[1], before[2], thr, nmin)
        if b0 < nmin:
            assert not conv.any()
        assert np.array_equal(after[2], before[2] + np.where(conv, 0, 8).astype(np.uint32))
        for k in (0, 1):  # converged pixels keep mean and M2 bit for bit
            assert np.array_equal(after[k][conv].view(np.uint32), before[k][conv].view(np.uint32))
        assert st["paths_skipped"] == 8 * int(conv.sum())
        assert st["paths"] + st["paths_skipped"] == W * H * 8
        total_skipped += st["paths_skipped"]
        before = after
    assert 0.1 * W * H * spp < total_skipped < 0.9 * W * H * spp, total_skipped
    img.close()
    scene.close()


def test_adaptive_render_matches_the_oracle(vp_ctx):
    spp, nmin = 64, 16
    g, cfg, envimg, scene, env, cam = workload(vp_ctx, "wavefront", spp, res=24)
    thr = threshold_for(vp_ctx, scene, env, cam, cfg, 0.5)
    cfg.adaptive_threshold, cfg.adaptive_min_samples = thr, nmin
    img = vp.ProgressiveImage(vp_ctx, cfg.image_width, cfg.image_height)
    img.accumulate(scene, env, cam, cfg, 0, spp)
    mean, _, cnt = state_of(img)
    osc = O.OracleScene.from_gaussians(g, sigma_multiplier=2.0)
    (omean, _, ocnt), _ = O.render_welford(osc, O.OracleEnv(envimg), O.camera16(cam, cfg.image_width,
                                                                                    cfg.image_height), cfg)
    same = cnt == ocnt
    assert np.mean(same) >= 0.9, np.mean(same)
    assert abs(int(cnt.sum()) - int(ocnt.sum())) <= 0.03 * ocnt.sum()
    assert 0 < np.sum(cnt < spp) < cnt.size
    scale = float(omean.mean())
    rel = np.abs(mean - omean)[same] / np.maximum(np.abs(omean[same]), 0.05 * scale)
    assert np.mean(rel < 1e-3) >= 0.95
    img.close()
    scene.close()


def test_adaptive_image_converges_to_the_full_render(vp_ctx):
    """Skipping converged pixels leaves the estimate unbiased up to the stopping rule: the adaptive
    image's error against a 4x-sample render stays within 1.5x of the full-spp image's, with
    fewer paths."""
    spp = 64
    g, cfg, _, scene, env, cam = workload(vp_ctx, "wavefront", spp * 4, res=32)
    W = H = cfg.image_width
    ref = vp.ProgressiveImage(vp_ctx, W, H)
    ref.accumulate(scene, env, cam, cfg, 0, spp * 4)
    truth = ref.read()[..., :3]
    full = vp.ProgressiveImage(vp_ctx, W, H)
    full.accumulate(scene, env, cam, cfg, 0, spp)
    cfg.adaptive_threshold = threshold_for(vp_ctx, scene, env, cam, cfg, 0.5, after=32)
    cfg.adaptive_min_samples = 32
    ada = vp.ProgressiveImage(vp_ctx, W, H)
    st = ada.accumulate(scene, env, cam, cfg, 0, spp)
    assert st["paths_skipped"] > 0
    err_full = np.sqrt(np.mean((full.read()[..., :3] - truth) ** 2))
    err_ada = np.sqrt(np.mean((ada.read()[..., :3] - truth) ** 2))
    assert err_ada < 1.5 * err_full, (err_ada, err_full)
    for im in (ref, full, ada):
        im.close()
    scene.close()


def test_adaptive_errors(vp_ctx):
    g, cfg, _, scene, env, cam = workload(vp_ctx, "wavefront", 16, res=8)
    img = vp.ProgressiveImage(vp_ctx, 8, 8)
    for bad in (-0.5, float("nan"), float("inf")):
        cfg.adaptive_threshold = bad
        with pytest.raises(vp.VpError, match="adaptive_threshold"):
            img.accumulate(scene, env, cam, cfg, 0, 8)
    img.clear()
    cfg.adaptive_threshold = 0.0
    img.accumulate(scene, env, cam, cfg, 0, 8)  # keeps no M2
    with pytest.raises(vp.VpError, match="M2"):
        img.read_welford()
    assert np.all(img.read_welford(m2=False)[1] == 8)
    cfg.adaptive_threshold = 0.2
    with pytest.raises(vp.VpError, match="M2"):
        img.accumulate(scene, env, cam, cfg, 8, 8)
    img.clear()
    img.accumulate(scene, env, cam, cfg, 0, 8)
    m2, cnt = img.read_welford()
    assert np.all(cnt == 8) and np.all(m2 >= 0.0)
    fresh = vp.ProgressiveImage(vp_ctx, 8, 8)
    m2, cnt = fresh.read_welford()
    assert not m2.any() and not cnt.any()
    fresh.close()
    img.close()
    scene.close()
