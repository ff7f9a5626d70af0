"""CPU: the oracle against the golden vectors of the reference's own code (tests/golden/), the
published PCG32 test vector, and the closed forms the reference's validation scripts use."""
import json
import math
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from volprim_b200 import scenes

GOLDEN = json.loads((Path(__file__).resolve().parent / "golden" / "reference_pin.json").read_text())


def f(bits):
    return np.asarray(bits, np.uint32).view(np.float32)


def test_pcg32_published_vector():
    g = GOLDEN["pcg32"]
    assert O.pcg32(g["seed"], g["sequence"], 6).tolist() == g["outputs"]


def test_primitive_records_match_reference():
    """Primitive constructor (primitive.h:70-87): conjugate quaternion, 1/scale, density norm,
    inv-CDF factor -- bit for bit."""
    for case in GOLDEN["primitives"]:
        sc = O.OracleScene(f(case["mean"])[None], f(case["scale"])[None], f(case["quat_wxyz"])[None],
                           f([case["density"]]), f(case["albedo"])[None])
        got = sc.records[0].view(np.uint32).tolist()
        assert got == case["record"], case


def test_whitening_and_containment_match_reference():
    for case in GOLDEN["primitives"]:
        sc = O.OracleScene(f(case["mean"])[None], f(case["scale"])[None], f(case["quat_wxyz"])[None],
                           f([case["density"]]), f(case["albedo"])[None])
        for t in case["transforms"]:
            got = sc.transform(0, f(t["pos"]), f(t["dir"])).view(np.uint32).tolist()
            assert got == t["out"]


def test_camera_matches_reference():
    import volprim_b200 as vp
    for c in GOLDEN["cameras"]:
        cam = vp.Camera(tuple(f(c["eye"])), tuple(f(c["lookat"])), tuple(f(c["up"])), float(f([c["vfov"]])[0]),
                        float(f([c["ortho_height"]])[0]), bool(c["orthographic"]))
        got = O.camera16(cam, c["width"], c["height"]).view(np.uint32).tolist()
        assert got == c["out"], c["name"]


def test_morton_matches_reference():
    m = GOLDEN["morton"]
    for c in m["cases"]:
        assert O.morton3d(f(c["pos"]), f(m["scene_min"]), f(m["inv_extent"])) == c["code"]


def test_single_gaussian_closed_form():
    """experiments/mitsuba-reference/single_gaussian_analytic.py:78-80 with the 3-sigma
    truncation the renderer integrates: tau(d) = M/(2 pi) e^{-d^2/2} erf(sqrt((9 - d^2)/2))."""
    sg = GOLDEN["single_gaussian"]
    d = np.asarray(sg["d"], np.float32)
    sc = O.OracleScene(np.zeros((1, 3)), np.ones((1, 3)), np.array([[1.0, 0, 0, 0]]), np.array([sg["mass"]]))
    o = np.stack([d, np.zeros_like(d), np.full_like(d, -5.0)], 1)
    dirs = np.tile([0.0, 0.0, 1.0], (len(d), 1))
    _, tau = sc.transmittance_fp64(o, dirs)
    dd = d.astype(np.float64)
    ref = sg["mass"] / (2 * math.pi) * np.exp(-dd ** 2 / 2) * np.array([math.erf(math.sqrt((9 - x * x) / 2)) for x in dd])
    np.testing.assert_allclose(tau, ref, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(tau, sg["tau"], rtol=1e-6)  # golden d values before float32 rounding


def test_fp32_restatement_tracks_fp64():
    """The FP32 reference-order transmittance (compute_transmittance_to_env) against the FP64 sum."""
    g = scenes.absorption_gaussians(256, 0)
    sc = O.OracleScene.from_gaussians(g)
    rng = np.random.default_rng(0)
    o = rng.normal(size=(3000, 3))
    o = (3.5 * o / np.linalg.norm(o, axis=1, keepdims=True)).astype(np.float32)
    d = rng.uniform(-0.7, 0.7, (3000, 3)) - o
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    T64, tau = sc.transmittance_fp64(o, d)
    T32 = sc.transmittance_fp32(o, d).astype(np.float64)
    sel = tau < 20
    assert (tau > 1).sum() > 300
    np.testing.assert_allclose(T32[sel], T64[sel], rtol=5e-3, atol=1e-7)


def test_env_tables():
    """Reference CDF (environment_map.h:45-101) and the alias tables give the same texel
    distribution, proportional to luminance x sin(theta)."""
    env = O.OracleEnv(scenes.procedural_env(64, 32, sun_radiance=100.0, sun_radius_deg=6.0))
    t = env.tables()
    W, H = 64, 32
    joint = t["joint"].reshape(H, W).astype(np.float64)
    p_true = joint / joint.sum()
    assert abs(t["marg_cdf"][-1] - 1.0) < 1e-6
    assert np.allclose(t["cond_cdf"].reshape(H, W)[:, -1], 1.0, atol=1e-6)
    # probability implied by the alias tables
    pm = np.zeros(H)
    for i in range(H):
        pm[i] += t["alias_marg_p"][i] / H
        pm[t["alias_marg_a"][i]] += (1 - t["alias_marg_p"][i]) / H
    pc = np.zeros((H, W))
    cp, ca = t["alias_cond_p"].reshape(H, W), t["alias_cond_a"].reshape(H, W)
    for v in range(H):
        for u in range(W):
            pc[v, u] += cp[v, u] / W
            pc[v, ca[v, u]] += (1 - cp[v, u]) / W
    np.testing.assert_allclose(pm[:, None] * pc, p_true, rtol=1e-5, atol=1e-9)
    # and the reference CDF's texel probabilities
    marg = np.diff(np.concatenate([[0.0], t["marg_cdf"].astype(np.float64)]))
    cond = np.diff(np.concatenate([np.zeros((H, 1)), t["cond_cdf"].reshape(H, W).astype(np.float64)], 1), axis=1)
    np.testing.assert_allclose(marg[:, None] * cond, p_true, rtol=1e-4, atol=1e-7)


def test_reference_morton_order_is_used():
    g = scenes.absorption_gaussians(64, 3)
    sc = O.OracleScene.from_gaussians(g)
    order = sc.order()
    assert sorted(order.tolist()) == list(range(64))
    c = g.mean.astype(np.float32)
    mn, mx = c.min(0), c.max(0)
    inv = (1.0 / np.maximum(mx - mn, 1e-30)).astype(np.float32)
    codes = [O.morton3d(c[i], mn, inv) for i in order]
    assert codes == sorted(codes)


def test_oracle_furnace():
    """White furnace on the oracle itself (albedo 1, unit environment)."""
    import volprim_b200 as vp
    rng = np.random.default_rng(7)
    n = 60
    g = vp.Gaussians(rng.uniform(-0.5, 0.5, (n, 3)), np.exp(rng.normal(math.log(0.2), 0.3, (n, 3))),
                     scenes.uniform_quaternions(rng, n), np.exp(rng.normal(0, 0.5, n)), np.ones((n, 3)))
    cfg = vp.Config(num_samples_per_pixel=64, image_width=16, image_height=16, seed=1, hg_g=0.0, max_bounces=512)
    sc = O.OracleScene.from_gaussians(g, sigma_multiplier=0.05)
    img, _ = O.render(sc, O.OracleEnv.constant(), O.camera16(scenes.negz_camera(3.0, 40.0), 16, 16), cfg,
                      rng_mode="sequential")
    sem = img.std() / math.sqrt(img.size)
    assert abs(img.mean() - 1.0) < max(5 * sem, 2e-3)


@pytest.mark.skipif(O.ref_lib() is None, reason="reference sources not present (pin library not built)")
def test_live_reference_pin_random():
    """Where the reference sources are mounted: random Gaussians and cameras, oracle vs the
    reference's own compiled headers, bit for bit."""
    R = O.ref_lib()
    rng = np.random.default_rng(11)
    out = np.empty(20, np.float32)
    for _ in range(200):
        m = rng.uniform(-3, 3, 3).astype(np.float32)
        s = np.exp(rng.normal(-2, 1, 3)).astype(np.float32)
        q = rng.normal(size=4).astype(np.float32)
        a = rng.uniform(0, 1, 3).astype(np.float32)
        M = np.float32(np.exp(rng.normal()))
        R.ref_primitive(O._p(m), O._p(s), O._p(q), O._p(a), float(M), O._p(out))
        sc = O.OracleScene(m[None], s[None], q[None], np.array([M]), a[None])
        assert sc.records[0].view(np.uint32).tolist() == out.view(np.uint32).tolist()


ADAPTIVE = GOLDEN["adaptive"]


def test_adaptive_constants_match_reference():
    """ENABLE_ADAPTIVE_SAMPLING, ADAPTIVE_MIN_SAMPLES, ADAPTIVE_THRESHOLD and
    ADAPTIVE_MIN_LUMINANCE (device/core/constants.cuh:196-211): the render defaults keep the
    reference's (off, 32), and the test's luminance floor is the reference's 1e-6f."""
    import ctypes as C
    from volprim_b200 import _capi
    p = _capi.vp_render_params()
    _capi.check(_capi.lib.vp_render_params_default(C.byref(p)))
    assert ADAPTIVE["enable"] is False
    assert p.adaptive_min_samples == ADAPTIVE["min_samples"] == 32
    assert np.float32(p.adaptive_threshold).view(np.uint32) == ADAPTIVE["threshold"]
    assert np.float32(1e-6).view(np.uint32) == ADAPTIVE["min_luminance"]


def test_welford_matches_reference():
    """The oracle's Welford step against the reference's own float3 operators (raygen.cuh:214-222),
    bit for bit, over heavy-tailed radiance sequences."""
    io = np.empty(6, np.float32)
    for case in ADAPTIVE["welford"]:
        L = f(case["L"]).reshape(-1, 3)
        io[:] = 0.0
        for k in range(L.shape[0]):
            O.lib().or_welford_step(O._p(np.ascontiguousarray(L[k])), k + 1, O._p(io))
        assert io.view(np.uint32).tolist() == case["out"], L.shape


def test_adaptive_test_matches_reference():
    """The oracle's convergence test decides err_max < threshold on the reference's own statistic
    (raygen.cuh:56-65): not converged at threshold = err_max, converged one ulp above it, never
    converged when the reference's max is NaN (a rounding-negative M2 in the last channel), and
    the NaN of the first channel dropped as the reference's `a > b ? a : b` drops it."""
    seen_nan = 0
    for case in ADAPTIVE["errors"]:
        mean, m2, n = f(case["mean"]), f(case["m2"]), case["count"]
        err = f(case["err"])[3]
        at = O.adaptive_converged(mean[None], m2[None], [n], float(err), 0)[0] if np.isfinite(err) else None
        if not np.isfinite(err):
            seen_nan += 1
            for thr in (1e-3, 1.0, 1e30):
                assert not O.adaptive_converged(mean[None], m2[None], [n], thr, 0)[0]
            continue
        above = float(np.nextafter(err, np.float32(np.inf)))
        assert not at, case
        assert O.adaptive_converged(mean[None], m2[None], [n], above, 0)[0], case
        # below the minimum sample count the test never passes (raygen.cuh:55)
        assert not O.adaptive_converged(mean[None], m2[None], [n], above, n + 1)[0]
    assert seen_nan == 1


def test_oracle_welford_render_and_adaptive_batches():
    """The oracle's progressive render: its mean and M2 are those of the per-sample radiances, and
    with adaptive sampling a pixel takes a batch exactly when its state before the batch fails the
    test."""
    import volprim_b200 as vp
    rng = np.random.default_rng(3)
    n = 40
    g = vp.Gaussians(rng.uniform(-0.5, 0.5, (n, 3)), np.exp(rng.normal(math.log(0.2), 0.3, (n, 3))),
                     scenes.uniform_quaternions(rng, n), np.exp(rng.normal(0, 0.5, n)),
                     rng.uniform(0.3, 0.9, (n, 3)))
    W = H = 8
    cfg = vp.Config(num_samples_per_pixel=48, image_width=W, image_height=H, seed=4, hg_g=0.3, max_bounces=16,
                    batch_spp=8)
    sc = O.OracleScene.from_gaussians(g, sigma_multiplier=2.0)
    env = O.OracleEnv.constant(1.0, 0.8, 0.6)
    c16 = O.camera16(scenes.negz_camera(2.5, 40.0), W, H)
    per = np.stack([O.render(sc, env, c16, cfg, s0=s, s1=s + 1)[0] for s in range(48)]).astype(np.float64)
    (mean, m2, cnt), _ = O.render_welford(sc, env, c16, cfg)
    assert np.all(cnt == 48)
    np.testing.assert_allclose(mean, per.mean(0), rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(m2, ((per - per.mean(0)) ** 2).sum(0), rtol=1e-4, atol=1e-6)
    cfg.adaptive_threshold, cfg.adaptive_min_samples = 0.6, 16
    state = None
    for b0 in range(0, 48, 8):
        before = None if state is None else tuple(a.copy() for a in state)
        state, _ = O.render_welford(sc, env, c16, cfg, state=state, s0=b0, s1=b0 + 8)
        if before is not None:
            conv = O.adaptive_converged(before[0], before[1], before[2], 0.6, 16)
            assert np.array_equal(state[2], before[2] + np.where(conv, 0, 8))
            assert np.array_equal(state[0][conv], before[0][conv])
    assert 0 < np.sum(state[2] < 48) < W * H, "some, not all, pixels must stop early"
