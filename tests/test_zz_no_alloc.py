"""GPU: vp_transmittance_static, the transmittance query for callers that cannot allocate device
memory (its scratch is a static device array), against vp_transmittance on the same rays.

Collected last (file name) so that a run stopping at the first failure has run every other test
first; it creates its own context and scene, so it also runs alone in a fresh process.
Tolerance: the transmittance tests' gate, |T - T_ref| <= 2e-5 T_ref + 1e-9.
"""
import math

import numpy as np
import pytest

import volprim_b200 as vp
from volprim_b200 import scenes
from volprim_b200._capi import VP_ENGINE_WARP, VP_PRECISION_ACCURATE, VP_PRECISION_FAST

pytestmark = pytest.mark.gpu


def _rays(seed, n):
    rng = np.random.default_rng(seed)
    o = rng.normal(size=(n, 3))
    o = 3.5 * o / np.linalg.norm(o, axis=1, keepdims=True)
    k = n // 3
    o[:k] = rng.uniform(-1, 1, (k, 3))  # a third start inside the cloud
    d = rng.uniform(-0.8, 0.8, (n, 3)) - o
    d[:k] = rng.normal(size=(k, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return o.astype(np.float32), d.astype(np.float32)


@pytest.fixture(scope="module")
def scene():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ctx = vp.Context(0)
    rng = np.random.default_rng(21)
    n = 3000
    g = vp.Gaussians(rng.uniform(-1, 1, (n, 3)), np.exp(rng.normal(math.log(0.08), 0.4, (n, 3))),
                     scenes.uniform_quaternions(rng, n), np.exp(rng.normal(0.0, 0.5, n)))
    sc = vp.Scene(ctx, g)
    yield sc
    sc.close()
    ctx.close()


def test_static_matches_allocating_query_two_calls(scene):
    for call, (seed, n, prec) in enumerate([(1, 40000, VP_PRECISION_ACCURATE), (2, 65536, VP_PRECISION_FAST)]):
        o, d = _rays(seed, n)
        ref = scene.transmittance(o, d, precision=prec, engine=VP_ENGINE_WARP).astype(np.float64)
        got = scene.transmittance_static(o, d, precision=prec).astype(np.float64)
        assert (ref < 0.99).sum() > n // 10, "rays must cross Gaussians"
        assert np.all(np.abs(got - ref) <= 2e-5 * ref + 1e-9), f"call {call}"


def test_static_device_pointers(scene):
    import torch
    o, d = _rays(3, 5000)
    ref = scene.transmittance(o, d, precision=VP_PRECISION_ACCURATE, engine=VP_ENGINE_WARP).astype(np.float64)
    got = scene.transmittance_static(torch.from_numpy(o).cuda(), torch.from_numpy(d).cuda(),
                                     precision=VP_PRECISION_ACCURATE).cpu().numpy().astype(np.float64)
    assert np.all(np.abs(got - ref) <= 2e-5 * ref + 1e-9)


def test_static_rejects_more_rays_than_its_scratch(scene):
    o, d = _rays(4, 65537)
    with pytest.raises(vp.VpError, match="at most 65536 rays"):
        scene.transmittance_static(o, d)


def test_static_waits_for_torch_stream(scene):
    """float64, non-contiguous CUDA inputs: their float32 copies are made by kernels on torch's
    stream, queued behind a busy-wait, so the query must wait for that stream before it reads."""
    import torch
    o, d = _rays(5, 8000)
    ref = scene.transmittance(o, d, precision=VP_PRECISION_FAST, engine=VP_ENGINE_WARP).astype(np.float64)
    o64 = torch.from_numpy(np.repeat(o.astype(np.float64), 2, axis=1)).cuda()[:, ::2]
    d64 = torch.from_numpy(np.repeat(d.astype(np.float64), 2, axis=1)).cuda()[:, ::2]
    assert not o64.is_contiguous()
    for _ in range(2):
        torch.cuda._sleep(20_000_000)
        got = scene.transmittance_static(o64, d64, precision=VP_PRECISION_FAST).cpu().numpy().astype(np.float64)
        assert np.all(np.abs(got - ref) <= 2e-5 * ref + 1e-9)
