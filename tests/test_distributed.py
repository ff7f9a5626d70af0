"""CPU, world size 2 over gloo: the sample sharding and the final image combination of the
multi-GPU path.  Each rank renders its sample range with the oracle (the CPU checker) and the
ranks combine with volprim_b200.distributed.combine; the result must equal the single-process
render over all samples."""
import math
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _workload():
    import volprim_b200 as vp
    from volprim_b200 import scenes
    rng = np.random.default_rng(3)
    n = 40
    g = vp.Gaussians(rng.uniform(-0.5, 0.5, (n, 3)), np.exp(rng.normal(math.log(0.15), 0.3, (n, 3))),
                     scenes.uniform_quaternions(rng, n), np.exp(rng.normal(0, 0.5, n)), np.full((n, 3), 0.8))
    cfg = vp.Config(num_samples_per_pixel=8, image_width=12, image_height=10, seed=5, hg_g=0.3, max_bounces=32)
    return g, cfg, scenes.negz_camera(3.0, 40.0)


def _rank_main(rank, world, port, out_path):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    sys.path[:0] = [str(root / "cuda-volprim_b200"), str(root / "oracle")]
    import oracle as O
    from volprim_b200 import distributed as D
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        g, cfg, cam = _workload()
        spp_per_rank = cfg.num_samples_per_pixel // world
        s0, cnt = D.sample_range(rank, world, spp_per_rank)
        sc = O.OracleScene.from_gaussians(g, sigma_multiplier=2.0)
        img, _ = O.render(sc, O.OracleEnv.constant(), O.camera16(cam, cfg.image_width, cfg.image_height), cfg,
                          s0=s0, s1=s0 + cnt, rng_mode="keyed", threads=1)
        comb = D.combine(torch.from_numpy(img.astype(np.float64)), cnt)
        if rank == 0:
            np.save(out_path, comb.numpy())
    finally:
        dist.destroy_process_group()


def test_sample_range():
    from volprim_b200 import distributed as D
    assert [D.sample_range(r, 4, 64) for r in range(4)] == [(0, 64), (64, 64), (128, 64), (192, 64)]
    with pytest.raises(ValueError):
        D.sample_range(4, 4, 64)


def test_two_rank_render_equals_single_process(tmp_path):
    import oracle as O
    port = _free_port()
    out = str(tmp_path / "combined.npy")
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    combined = np.load(out)
    g, cfg, cam = _workload()
    sc = O.OracleScene.from_gaussians(g, sigma_multiplier=2.0)
    full, _ = O.render(sc, O.OracleEnv.constant(), O.camera16(cam, cfg.image_width, cfg.image_height), cfg,
                       rng_mode="keyed", threads=1)
    assert full.mean() > 0.01
    np.testing.assert_allclose(combined, full, rtol=1e-5, atol=1e-7)
