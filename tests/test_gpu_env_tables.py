"""GPU: the environment sampling tables the device builds in FP64 (vp_env.cu), read back with
vp_env_read_tables, on the 2048x1024 procedural environment of the showcase workload (sky
gradient, a 0.5-degree sun of 1e4 relative radiance, dim ground).

The reference samples texels in proportion to luminance x sin(theta at the row centre) through
an FP32 2-D CDF (EnvironmentMap::buildCdf, include/thesis/host/params/environment_map.h:45-101).
Its FP64 restatement here is p_true = w / sum(w), w = (0.2126 r + 0.7152 g + 0.0722 b) sin(theta).

Bounds:
  * every texel's probability implied by the device's alias tables is within 1e-6 relative of
    p_true (the FP64 tables rounded to FP32 give 9e-8 on this map), including the 29 sun texels
    that hold a third of the mass;
  * the reference's own FP32 CDF on the same map is within 5e-2 relative of p_true (3.4e-2 worst,
    on the faintest texels, where its cumulative sums have run out of bits) -- the alias tables
    are the tighter of the two;
  * the tables are well formed: probabilities in [0, 1], aliases inside their row / the map.
"""
import numpy as np
import pytest

import oracle as O
import volprim_b200 as vp
from volprim_b200 import scenes

pytestmark = pytest.mark.gpu


def implied_texel_probability(cond_prob, cond_alias, marg_prob, marg_alias):
    """Probability of each texel under two alias draws (row, then texel within the row)."""
    H, W = cond_prob.shape
    pm = marg_prob.astype(np.float64) / H
    pm = pm + np.bincount(marg_alias, weights=(1.0 - marg_prob.astype(np.float64)) / H, minlength=H)
    rows = np.repeat(np.arange(H, dtype=np.int64), W)
    pc = cond_prob.reshape(-1).astype(np.float64) / W
    pc = pc + np.bincount(rows * W + cond_alias.reshape(-1), weights=(1.0 - cond_prob.reshape(-1).astype(np.float64)) / W,
                          minlength=H * W)
    return pm[:, None] * pc.reshape(H, W)


@pytest.fixture(scope="module")
def showcase_env(vp_ctx):
    rgb = scenes.procedural_env(2048, 1024)
    env = vp.Environment(vp_ctx, rgb=rgb)
    yield rgb, env
    env.close()


def test_showcase_alias_tables_match_fp64_distribution(showcase_env):
    rgb, env = showcase_env
    t = env.tables()
    H, W = rgb.shape[:2]
    assert t["cond_prob"].shape == (H, W) and t["marg_prob"].shape == (H,)
    assert np.all((t["cond_prob"] >= 0) & (t["cond_prob"] <= 1)) and np.all((t["marg_prob"] >= 0) & (t["marg_prob"] <= 1))
    assert t["cond_alias"].max() < W and t["marg_alias"].max() < H
    lum = 0.2126 * rgb[..., 0].astype(np.float64) + 0.7152 * rgb[..., 1] + 0.0722 * rgb[..., 2]
    w = lum * np.sin((np.arange(H) + 0.5) / H * np.pi)[:, None]
    np.testing.assert_allclose(t["joint"], w, rtol=1e-6, atol=0)
    assert abs(t["total"] - w.sum()) <= 1e-6 * w.sum()
    p_true = w / w.sum()
    p = implied_texel_probability(t["cond_prob"], t["cond_alias"], t["marg_prob"], t["marg_alias"])
    rel = np.abs(p - p_true) / p_true
    sun = p_true > 1e-4
    assert sun.sum() > 10 and p_true[sun].sum() > 0.3, "the sun lobe must be resolved"
    assert rel.max() <= 1e-6, f"worst texel {rel.max():.3e} (sun {rel[sun].max():.3e})"
    # the reference's own FP32 CDF on the same map, through the oracle's restatement
    ot = O.OracleEnv(rgb).tables()
    marg = np.diff(np.concatenate([[0.0], ot["marg_cdf"].astype(np.float64)]))
    cond = np.diff(np.concatenate([np.zeros((H, 1)), ot["cond_cdf"].reshape(H, W).astype(np.float64)], 1), axis=1)
    rel_cdf = np.abs(marg[:, None] * cond - p_true) / p_true
    assert rel_cdf.max() <= 5e-2 and rel.max() < rel_cdf.max()


def test_constant_environment_tables(vp_ctx):
    env = vp.Environment(vp_ctx, constant=(1.0, 1.0, 1.0))
    t = env.tables()
    assert t["cond_prob"].shape == (1, 2)
    p = implied_texel_probability(t["cond_prob"], t["cond_alias"], t["marg_prob"], t["marg_alias"])
    np.testing.assert_allclose(p, 0.5, rtol=1e-7)
    env.close()
