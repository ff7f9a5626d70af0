"""GPU: the serving loop (vp_server_*) -- resident scenes, memory-budget admission, continuous
batching of mixed requests into shared wavefront launches under a CUDA graph.

Tolerances.  A served request's paths run the offline engine's per-path code with the same PCG32
stream per (pixel, sample), so each path's sample is the offline one; the per-pixel mean differs
only by the order of its FP32 sums (atomic adds in completion order vs the offline Welford mean in
sample order):
  served vs served (alone vs in a mix, graph vs no graph):  |a - b| <= 1e-5 |b| + 1e-6
  served vs offline vp_render (wavefront engine): >= 99% of pixels within 1e-5 relative + 1e-6 and
  mean |a - b| / mean |b| < 1e-5 (the two kernels may contract FP32 operations differently, which
  can flip a rare roulette or acceptance decision)
"""
import numpy as np
import pytest

import volprim_b200 as vp
from volprim_b200 import scenes
from volprim_b200.serving import Server, make_trace, run_trace

pytestmark = pytest.mark.gpu


def close(a, b, rel=1e-5, abs_=1e-6):
    return np.abs(a - b) <= rel * np.abs(b) + abs_


@pytest.fixture(scope="module")
def world(vp_ctx):
    gs = [scenes.showcase_gaussians(n, seed) for n, seed in ((20_000, 1), (60_000, 2))]
    env_img = scenes.procedural_env(256, 128, sun_radiance=200.0, sun_radius_deg=3.0)
    scs = [vp.Scene(vp_ctx, g, 7.5) for g in gs]
    envs = [vp.Environment(vp_ctx, rgb=env_img) for _ in gs]
    yield {"scenes": scs, "envs": envs}
    for e in envs:
        e.close()
    for s in scs:
        s.close()


def new_server(vp_ctx, world, **kw):
    srv = Server(vp_ctx, **{"path_slots": 1 << 18, "max_requests": 64, **kw})
    for s, e in zip(world["scenes"], world["envs"]):
        srv.add_scene(s, e)
    return srv


def drain(srv, limit=100000):
    done = []
    for _ in range(limit):
        srv.step()
        done += srv.poll()
        st = srv.stats()
        if st["active"] == 0 and st["pending"] == 0:
            return done
    raise AssertionError("server did not drain")


def requests(seed, n):
    tr = make_trace(seed, n, rate=0.0, n_scenes=2, resolutions=(32, 48, 64), spps=(1, 4, 8))
    return tr


def test_served_request_matches_offline_render(vp_ctx, world):
    srv = new_server(vp_ctx, world)
    r = requests(3, 1)[0]
    rid = srv.submit(r.scene_id, r.camera, r.config)
    assert rid in drain(srv)
    got = srv.result(rid)[..., :3]
    cfg = vp.Config(**{**r.config.__dict__, "engine": "wavefront"})
    ref = vp.Renderer(cfg, world["scenes"][r.scene_id], r.camera, env=world["envs"][r.scene_id], ctx=vp_ctx).render()[..., :3]
    assert ref.mean() > 1e-3
    assert np.mean(close(got, ref)) >= 0.99
    assert np.abs(got - ref).mean() / np.abs(ref).mean() < 1e-5
    srv.close()


def test_same_result_alone_and_in_the_mix(vp_ctx, world):
    """Request X rendered alone, then inside a mix where other requests of both scenes and other
    resolutions and sample counts are already running when X arrives, and more arrive after it."""
    mix = requests(5, 12)
    x = mix[6]
    alone = new_server(vp_ctx, world)
    rid = alone.submit(x.scene_id, x.camera, x.config)
    drain(alone)
    img_alone = alone.result(rid)
    alone.close()

    srv = new_server(vp_ctx, world, iterations_per_step=2)
    ids = [srv.submit(r.scene_id, r.camera, r.config) for r in mix[:6]]
    srv.step()
    srv.step()
    assert srv.stats()["active"] >= 2, "earlier requests must be on the GPU when X arrives"
    ids.append(srv.submit(x.scene_id, x.camera, x.config))
    srv.step()
    ids += [srv.submit(r.scene_id, r.camera, r.config) for r in mix[7:]]
    overlapped = False
    done = []
    for _ in range(100000):
        srv.step()
        st = srv.stats()
        done += srv.poll()
        if ids[6] not in done and st["active"] >= 2:
            overlapped = True
        if st["active"] == 0 and st["pending"] == 0:
            break
    assert sorted(done) == sorted(ids)
    assert overlapped
    img_mix = srv.result(ids[6])
    assert np.all(close(img_mix, img_alone)), float(np.abs(img_mix - img_alone).max())
    # every other request of the mix equals its own offline render
    for r, rid in zip(mix, ids):
        if rid == ids[6]:
            continue
        got = srv.result(rid)[..., :3]
        cfg = vp.Config(**{**r.config.__dict__, "engine": "wavefront"})
        ref = vp.Renderer(cfg, world["scenes"][r.scene_id], r.camera, env=world["envs"][r.scene_id],
                          ctx=vp_ctx).render()[..., :3]
        assert np.mean(close(got, ref)) >= 0.99
    srv.close()


def test_graph_and_direct_launches_agree(vp_ctx, world):
    reqs = requests(7, 5)
    out = {}
    for g in (True, False):
        srv = new_server(vp_ctx, world, use_graph=g)
        ids = [srv.submit(r.scene_id, r.camera, r.config) for r in reqs]
        drain(srv)
        out[g] = [srv.result(i) for i in ids]
        srv.close()
    for a, b in zip(out[True], out[False]):
        assert np.all(close(a, b))


def test_lanes_agree(vp_ctx, world):
    """Two lanes (independent path pools on their own streams, each request in one of them) give
    every request the output one lane gives it."""
    reqs = requests(13, 10)
    out = {}
    for lanes in (1, 2):
        srv = new_server(vp_ctx, world, lanes=lanes)
        ids = [srv.submit(r.scene_id, r.camera, r.config) for r in reqs]
        assert sorted(drain(srv)) == sorted(ids)
        out[lanes] = [srv.result(i) for i in ids]
        srv.close()
    for a, b in zip(out[1], out[2]):
        assert np.all(close(a, b))


def test_schedules(vp_ctx, world):
    """Every schedule gives the same images; under FAIR and SRPT a small request submitted after
    a large one (more paths than the slot pool) completes first."""
    big = make_trace(15, 1, rate=0.0, n_scenes=1, resolutions=(256,), spps=(8,))[0]
    small = make_trace(16, 1, rate=0.0, n_scenes=1, resolutions=(32,), spps=(1,))[0]
    imgs = {}
    for sched in ("fair", "fifo", "srpt"):
        srv = new_server(vp_ctx, world, schedule=sched, iterations_per_step=2)
        ib = srv.submit(big.scene_id, big.camera, big.config)
        isml = srv.submit(small.scene_id, small.camera, small.config)
        order = drain(srv)
        if sched in ("fair", "srpt"):
            assert order.index(isml) < order.index(ib), sched
        imgs[sched] = (srv.result(ib), srv.result(isml))
        srv.close()
    for sched in ("fifo", "srpt"):
        for a, b in zip(imgs[sched], imgs["fair"]):
            assert np.all(close(a, b)), sched


def test_srpt_aging(vp_ctx, world):
    """SRPT with aging gives the same images as plain SRPT; a negative aging is refused."""
    reqs = requests(21, 6)
    out = {}
    for aging in (0.0, 1.0):
        srv = new_server(vp_ctx, world, schedule="srpt", srpt_aging=aging, iterations_per_step=2)
        ids = [srv.submit(r.scene_id, r.camera, r.config) for r in reqs]
        assert sorted(drain(srv)) == sorted(ids)
        out[aging] = [srv.result(i) for i in ids]
        srv.close()
    for a, b in zip(out[0.0], out[1.0]):
        assert np.all(close(a, b))
    with pytest.raises(vp.VpError, match="srpt_aging"):
        new_server(vp_ctx, world, schedule="srpt", srpt_aging=-1.0)


def test_admission_respects_the_memory_budget(vp_ctx, world):
    probe = new_server(vp_ctx, world)
    fixed = probe.stats()["bytes_in_use"]
    probe.close()
    reqs = make_trace(9, 8, rate=0.0, n_scenes=2, resolutions=(64,), spps=(1, 4, 8))
    per = 64 * 64 * 16 * 2  # each request: accumulator + host output staging
    srv = new_server(vp_ctx, world, memory_budget_bytes=fixed + 2 * per)
    ids = [srv.submit(r.scene_id, r.camera, r.config) for r in reqs]
    max_active = 0
    for _ in range(100000):
        srv.step()
        st = srv.stats()
        max_active = max(max_active, st["active"])
        assert st["bytes_in_use"] <= fixed + 2 * per
        if st["active"] == 0 and st["pending"] == 0:
            break
    assert 1 <= max_active <= 2
    assert srv.stats()["completed"] == len(reqs)
    solo = new_server(vp_ctx, world)
    for r, rid in zip(reqs, ids):
        sid = solo.submit(r.scene_id, r.camera, r.config)
        drain(solo)
        assert np.all(close(srv.result(rid), solo.result(sid)))
    solo.close()
    srv.close()


def test_real_time_trace(vp_ctx, world):
    tr = make_trace(11, 24, rate=40.0, n_scenes=2, resolutions=(32, 64, 96), spps=(1, 4, 16))
    srv = new_server(vp_ctx, world)
    res = run_trace(srv, tr)
    assert all(v is not None and v > 0 for v in res["latency_s"])
    assert res["server"]["completed"] == len(tr)
    assert res["p99_s"] >= res["p50_s"] > 0
    srv.close()


def test_invalid_requests_raise(vp_ctx, world):
    srv = new_server(vp_ctx, world)
    r = requests(13, 1)[0]
    with pytest.raises(vp.VpError, match="unknown scene_id"):
        srv.submit(7, r.camera, r.config)
    bad = vp.Config(**{**r.config.__dict__, "max_bounces": 0})
    with pytest.raises(vp.VpError, match="max_bounces"):
        srv.submit(0, r.camera, bad)
    adaptive = vp.Config(**{**r.config.__dict__, "adaptive_threshold": 0.1})
    with pytest.raises(vp.VpError, match="adaptive sampling"):
        srv.submit(0, r.camera, adaptive)
    srv.close()
    tiny = new_server(vp_ctx, world)
    fixed = tiny.stats()["bytes_in_use"]
    tiny.close()
    small = new_server(vp_ctx, world, memory_budget_bytes=fixed + 1000)
    with pytest.raises(vp.VpError, match="memory budget"):
        small.submit(0, r.camera, r.config)
    small.close()


# -- host-side faults: cancellation and failed accumulator allocations ---------------------------

VP_ERROR_OUT_OF_MEMORY = -3


def solo_image(vp_ctx, world, r):
    solo = new_server(vp_ctx, world)
    sid = solo.submit(r.scene_id, r.camera, r.config)
    drain(solo)
    img = solo.result(sid)
    solo.close()
    return img


def test_cancel_queued_and_running_requests(vp_ctx, world):
    """A request cancelled while queued and one cancelled while its paths run: neither is ever
    delivered nor writes its output, the others finish with their solo results, and the table
    entries and memory come back."""
    reqs = make_trace(17, 3, rate=0.0, n_scenes=2, resolutions=(96,), spps=(16,))
    srv = new_server(vp_ctx, world, iterations_per_step=2)
    fixed = srv.stats()["bytes_in_use"]
    shape = (96, 96, 4)
    outs = [np.full(shape, -7.0, np.float32) for _ in reqs]
    ids = [srv.submit(r.scene_id, r.camera, r.config, out=o) for r, o in zip(reqs, outs)]
    srv.cancel(ids[2])  # still queued
    assert srv.stats()["pending"] == 2
    srv.step()
    srv.step()
    assert srv.stats()["active"] == 2
    srv.cancel(ids[0])  # admitted, paths in flight
    with pytest.raises(vp.VpError, match="already cancelled"):
        srv.cancel(ids[0])
    done = drain(srv)
    assert done == [ids[1]]
    st = srv.stats()
    assert st["cancelled"] == 2 and st["completed"] == 1 and st["active"] == 0
    assert st["bytes_in_use"] == fixed
    assert np.all(outs[0] == -7.0) and np.all(outs[2] == -7.0)
    assert np.all(close(srv.result(ids[1]), solo_image(vp_ctx, world, reqs[1])))
    for rid in (ids[1], ids[0], 12345):  # delivered, released after cancel, never submitted
        with pytest.raises(vp.VpError):
            srv.cancel(rid)
    # the freed entries and memory serve new requests
    rid = srv.submit(reqs[0].scene_id, reqs[0].camera, reqs[0].config)
    assert drain(srv) == [rid]
    assert np.all(close(srv.result(rid), solo_image(vp_ctx, world, reqs[0])))
    srv.close()


def test_cancel_releases_the_memory_budget(vp_ctx, world):
    probe = new_server(vp_ctx, world)
    fixed = probe.stats()["bytes_in_use"]
    probe.close()
    reqs = make_trace(19, 2, rate=0.0, n_scenes=2, resolutions=(64,), spps=(64,))
    per = 64 * 64 * 16 * 2
    srv = new_server(vp_ctx, world, memory_budget_bytes=fixed + per, iterations_per_step=2)
    ids = [srv.submit(r.scene_id, r.camera, r.config) for r in reqs]
    srv.step()
    assert srv.stats()["active"] == 1 and srv.stats()["pending"] == 1
    srv.cancel(ids[0])
    assert drain(srv) == [ids[1]]
    assert np.all(close(srv.result(ids[1]), solo_image(vp_ctx, world, reqs[1])))
    srv.close()


def test_failed_accumulator_allocation(vp_ctx, world):
    """Injected on the host: with nothing admitted the step reports out of memory and keeps the
    request queued; with a request admitted the new one waits; either way the server stays usable
    and the results are the solo ones."""
    reqs = requests(23, 3)
    srv = new_server(vp_ctx, world)
    srv.inject_alloc_failures(1)
    a = srv.submit(reqs[0].scene_id, reqs[0].camera, reqs[0].config)
    with pytest.raises(vp.VpError) as ei:
        srv.step()
    assert ei.value.status == VP_ERROR_OUT_OF_MEMORY
    st = srv.stats()
    assert st["alloc_failures"] == 1 and st["pending"] == 1 and st["active"] == 0
    srv.step()  # the retry succeeds
    assert srv.stats()["active"] == 1
    srv.inject_alloc_failures(1)
    b = srv.submit(reqs[1].scene_id, reqs[1].camera, reqs[1].config)
    srv.step()  # a is admitted: b waits instead of failing the step
    st = srv.stats()
    assert st["alloc_failures"] == 2 and st["pending"] == 1
    assert sorted(drain(srv)) == sorted([a, b])
    for rid, r in ((a, reqs[0]), (b, reqs[1])):
        assert np.all(close(srv.result(rid), solo_image(vp_ctx, world, r)))
    # a request stuck behind failing allocations can be cancelled
    srv.inject_alloc_failures(3)
    c = srv.submit(reqs[2].scene_id, reqs[2].camera, reqs[2].config)
    with pytest.raises(vp.VpError):
        srv.step()
    srv.cancel(c)
    srv.inject_alloc_failures(0)
    st = srv.stats()
    assert st["pending"] == 0 and st["cancelled"] == 1 and st["completed"] == 2
    srv.close()
