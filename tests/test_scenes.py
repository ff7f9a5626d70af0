"""CPU: the seeded workload generators (shapes, determinism, the stated distributions)."""
import math

import numpy as np

from volprim_b200 import scenes


def test_absorption_workload_distributions():
    w = scenes.absorption_256()
    g = w.gaussians
    assert g.mean.shape == (256, 3) and g.scale.shape == (256, 3) and g.quat_wxyz.shape == (256, 4)
    assert g.mean.min() >= -1 and g.mean.max() <= 1
    assert abs(np.log(g.scale).mean() - math.log(0.1)) < 0.05 and abs(np.log(g.scale).std() - 0.4) < 0.04
    assert abs(np.log(g.density).mean() - math.log(5.0)) < 0.1 and abs(np.log(g.density).std() - 0.5) < 0.06
    np.testing.assert_allclose(np.linalg.norm(g.quat_wxyz, axis=1), 1.0, atol=1e-6)
    assert np.all(g.albedo == 0)
    c = w.config
    assert (c.image_width, c.image_height, c.num_samples_per_pixel, c.seed) == (128, 128, 16, 0)
    assert w.camera.eye == (0.0, 0.0, -3.5) and w.camera.vfov_deg == 40.0
    assert w.paths == 128 * 128 * 16


def test_generators_are_deterministic():
    a, b = scenes.absorption_gaussians(64, 5), scenes.absorption_gaussians(64, 5)
    for x, y in ((a.mean, b.mean), (a.scale, b.scale), (a.quat_wxyz, b.quat_wxyz), (a.density, b.density)):
        assert np.array_equal(x, y)
    s1, s2 = scenes.showcase_gaussians(20000, 1), scenes.showcase_gaussians(20000, 1)
    assert np.array_equal(s1.mean, s2.mean)
    assert not np.array_equal(s1.mean, scenes.showcase_gaussians(20000, 2).mean)


def test_showcase_distributions():
    g = scenes.showcase_gaussians(50000, 0)
    assert np.all(g.mean[:, 0] >= -1) and np.all(g.mean[:, 0] <= 1)
    assert np.all(np.abs(g.mean[:, 1:]) <= 0.5)
    assert abs(np.log(g.scale).mean() - math.log(0.02)) < 0.02 and abs(np.log(g.scale).std() - 0.5) < 0.02
    assert abs(np.log(g.density).mean()) < 0.02 and abs(np.log(g.density).std() - 0.7) < 0.02
    assert np.all(g.albedo == np.float32(0.9))
    # means come only from where the value noise exceeds the threshold
    assert np.all(scenes.value_noise(g.mean[:2000].astype(np.float64), 0 + 7919) > 0.55)
    # uniform rotations: E[w^2] = 1/4
    assert abs((g.quat_wxyz[:, 0] ** 2).mean() - 0.25) < 0.01


def test_stress_distributions():
    g = scenes.stress_gaussians(40000, 0)
    assert abs(np.log(g.scale).mean() - math.log(0.05)) < 0.01 and abs(np.log(g.scale).std() - 0.3) < 0.01
    assert abs(np.log(g.density).mean() - math.log(2.0)) < 0.02
    assert np.all(g.albedo == np.float32(0.8))


def test_procedural_environment():
    env = scenes.procedural_env(256, 128, sun_radiance=1e4, sun_radius_deg=2.0)
    assert env.shape == (128, 256, 3) and env.dtype == np.float32
    assert env.max() >= 1e4 * 0.85 and np.isfinite(env).all() and env.min() > 0
    # the sun sits where the reference's lat-long mapping puts sun_dir
    s = np.array([0.7197, 0.4530, 0.5261])
    s /= np.linalg.norm(s)
    v, u = np.unravel_index(np.argmax(env[..., 0]), env.shape[:2])
    polar, theta = (v + 0.5) / 128 * math.pi, ((u + 0.5) / 256 - 0.5) * 2 * math.pi
    d = np.array([math.sin(polar) * math.cos(theta), math.cos(polar), math.sin(polar) * math.sin(theta)])
    assert np.dot(d, s) > math.cos(math.radians(3.0))
    # ground below the horizon is dim, sky above is brighter
    assert env[100:, :, 0].mean() < 0.1 < env[:50, :, 2].mean()


def test_validation_scenes_are_the_reference_runners():
    """Every geometric validation and stress scene of the reference's test runner
    (test/scenes/geometric_validation.cpp, compiled from the reference's source into the golden
    generator's pin library): same names, order and Gaussian counts, and the same float32 centre,
    rotation, scale, albedo and optical thickness bit for bit (digest of the rows)."""
    import hashlib
    import json
    from pathlib import Path

    import validation_scenes as VS
    golden = json.loads((Path(__file__).resolve().parent / "golden" / "reference_pin.json").read_text())
    want = golden["validation_scenes"]
    got = VS.all_scenes()
    assert [s.name for s in got] == [w["name"] for w in want]
    assert len(VS.validation_scenes()) == 36 and len(VS.stress_scenes()) == 7
    for s, w in zip(got, want):
        g = s.gaussians
        assert g.count == w["count"], s.name
        rows = np.concatenate([g.mean, g.quat_wxyz, g.scale, g.albedo, g.density[:, None]], 1).astype(np.float32)
        assert hashlib.sha256(np.ascontiguousarray(rows).tobytes()).hexdigest() == w["sha256"], s.name
