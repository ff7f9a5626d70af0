"""GPU: the absorption-plus-emission image (vp_render_emission) and its hand-written adjoint
(vp_render_emission_backward) on the differentiation workload -- 100k Gaussians with the 500k
showcase's distributions, RGB emission U[0,1], 4 cameras, 256x256, 8 spp, L2 loss against a
seeded render of perturbed parameters -- against the FP64 oracle (oracle/emission_oracle.py):

  forward   per pixel on 32x32 crops of every camera:  |L - L64| <= 1e-4 max(|L64|, 1e-2)
  autodiff  FP64 PyTorch autograd of the same closed form on a 32x32 crop of camera 0: every
            parameter group within 1e-3 relative (L2 norm over the group), and each parameter
            whose gradient exceeds 1e-2 of its group's largest within 1e-2 relative (FAST and
            ACCURATE adjoints)
  FD        FP64 central finite differences on 64 random parameters (the mean, log-scale,
            quaternion and density components of random visible Gaussians):
            |g - g_fd| <= 1e-3 |g_fd| + 1e-6 G, G = the largest |g_fd| of the 64 (FAST and
            ACCURATE adjoints).  The 3-sigma truncation gives tau a square-root kink where a ray
            grazes the ellipsoid; each step is kept below 2% of the parameter distance at which
            any ray first reaches it (a parameter whose step would fall below 1e-9 is skipped).
"""

import numpy as np
import pytest
import torch

import oracle as O
import emission_oracle as E
import volprim_b200 as vp
from volprim_b200 import scenes
from volprim_b200.emission import render_emission, render_emission_backward

pytestmark = pytest.mark.gpu

CROP = 32


@pytest.fixture(scope="module")
def c5(vp_ctx):
    w = scenes.emission_100k()
    cfg = w.config
    scene = vp.Scene(vp_ctx, w.gaussians, w.sigma_multiplier)
    scene.set_emission(w.emission)
    env = vp.Environment(vp_ctx, constant=w.env_constant)
    tg, te = scenes.perturbed(w)
    tscene = vp.Scene(vp_ctx, tg, w.sigma_multiplier)
    tscene.set_emission(te)
    targets = [render_emission(tscene, env, cam, cfg)[..., :3].astype(np.float64) for cam in w.cameras]
    tscene.close()
    imgs = [render_emission(scene, env, cam, cfg)[..., :3].astype(np.float64) for cam in w.cameras]
    osc = O.OracleScene.from_gaussians(w.gaussians, w.sigma_multiplier, use_bvh=True)
    yield {"w": w, "scene": scene, "env": env, "imgs": imgs, "targets": targets, "osc": osc}
    env.close()
    scene.close()


def crop_rays(w, k, x0, y0, size=CROP):
    cfg = w.config
    spp = cfg.num_samples_per_pixel
    ys, xs = np.mgrid[y0:y0 + size, x0:x0 + size]
    px = np.repeat(xs.reshape(-1), spp)
    py = np.repeat(ys.reshape(-1), spp)
    sm = np.tile(np.arange(spp), size * size)
    c16 = O.camera16(w.cameras[k], cfg.image_width, cfg.image_height)
    return O.camera_rays(c16, cfg.image_width, spp, cfg.seed, px, py, sm)


def oracle_pixels(c, k, x0, y0, size=CROP):
    """FP64 crop image (size, size, 3) from the C++ oracle's ray sums."""
    w = c["w"]
    spp = w.config.num_samples_per_pixel
    o, d = crop_rays(w, k, x0, y0, size)
    S, C = c["osc"].emission_sums(w.emission, o, d)
    env = torch.tensor(w.env_constant, dtype=torch.float64).expand(len(o), 3)
    L = E.radiance(torch.tensor(S), torch.tensor(C), env).numpy()
    return L.reshape(size * size, spp, 3).mean(1).reshape(size, size, 3)


def crop_origin(c, k):
    """A crop where the cloud covers the image (largest mean optical effect in a coarse grid)."""
    img = c["imgs"][k]
    H = img.shape[0]
    best, at = -1.0, (0, 0)
    for y0 in range(0, H - CROP + 1, CROP):
        for x0 in range(0, H - CROP + 1, CROP):
            v = float(np.abs(img[y0:y0 + CROP, x0:x0 + CROP] - 1.0).mean())
            if v > best:
                best, at = v, (x0, y0)
    return at


def zero_grads(n):
    return {"mean": np.zeros(3 * n, np.float32), "scale": np.zeros(3 * n, np.float32),
            "quat_wxyz": np.zeros(4 * n, np.float32), "density": np.zeros(n, np.float32),
            "emission": np.zeros(3 * n, np.float32)}


@pytest.mark.parametrize("k", [0, 1, 2, 3])
def test_forward_matches_fp64(c5, k):
    x0, y0 = crop_origin(c5, k)
    ref = oracle_pixels(c5, k, x0, y0)
    got = c5["imgs"][k][y0:y0 + CROP, x0:x0 + CROP]
    assert np.abs(ref - 1.0).max() > 0.05, "the crop must see the cloud"
    err = np.abs(got - ref)
    assert np.all(err <= 1e-4 * np.maximum(np.abs(ref), 1e-2)), float(err.max())


def test_forward_accurate_precision(c5, vp_ctx):
    w = c5["w"]
    cfg = vp.Config(**{**w.config.__dict__, "precision": "accurate"})
    img = render_emission(c5["scene"], c5["env"], w.cameras[0], cfg)[..., :3]
    x0, y0 = crop_origin(c5, 0)
    ref = oracle_pixels(c5, 0, x0, y0)
    err = np.abs(img[y0:y0 + CROP, x0:x0 + CROP] - ref)
    assert np.all(err <= 2e-5 * np.maximum(np.abs(ref), 1e-2)), float(err.max())


def test_adjoint_matches_fp64_autodiff_on_crop(c5):
    w = c5["w"]
    n = w.gaussians.count
    x0, y0 = crop_origin(c5, 0)
    target = torch.tensor(c5["targets"][0][y0:y0 + CROP, x0:x0 + CROP])
    p = E.params_from(w.gaussians, requires_grad=True)
    em = torch.tensor(w.emission, dtype=torch.float64, requires_grad=True)
    spp = w.config.num_samples_per_pixel
    o, d = crop_rays(w, 0, x0, y0)
    ri, gi = c5["osc"].ray_candidates(o, d)
    S, C = E.ray_sums(p, em, w.sigma_multiplier, torch.tensor(o, dtype=torch.float64),
                      torch.tensor(d, dtype=torch.float64), torch.tensor(ri), torch.tensor(gi), len(o))
    L = E.radiance(S, C, torch.tensor(w.env_constant, dtype=torch.float64).expand(len(o), 3))
    pix = L.reshape(CROP * CROP, spp, 3).mean(1).reshape(CROP, CROP, 3)
    loss = ((pix - target) ** 2).sum()
    loss.backward()
    # the same upstream gradient for the adjoint
    dl = np.zeros((w.config.image_height, w.config.image_width, 4), np.float32)
    dl[y0:y0 + CROP, x0:x0 + CROP, :3] = (2.0 * (pix.detach() - target)).numpy()
    ref = {"mean": p["mean"].grad.numpy().reshape(-1), "scale": p["log_scale"].grad.numpy().reshape(-1),
           "quat_wxyz": p["quat"].grad.numpy().reshape(-1), "density": p["density"].grad.numpy().reshape(-1),
           "emission": em.grad.numpy().reshape(-1)}
    for prec in ("fast", "accurate"):
        cfg = vp.Config(**{**w.config.__dict__, "precision": prec})
        g = zero_grads(n)
        render_emission_backward(c5["scene"], c5["env"], w.cameras[0], cfg, dl, g)
        for key, r in ref.items():
            got = g[key].astype(np.float64)
            assert np.abs(r).max() > 0, key
            rel = np.linalg.norm(got - r) / np.linalg.norm(r)
            assert rel <= 1e-3, (prec, key, rel)
            big = np.abs(r) > 1e-2 * np.abs(r).max()
            assert np.all(np.abs(got[big] - r[big]) <= 1e-2 * np.abs(r[big])), (prec, key)


def test_adjoint_matches_finite_differences(c5):
    w = c5["w"]
    cfg = w.config
    g = w.gaussians
    n = g.count
    W, H, spp = cfg.image_width, cfg.image_height, cfg.num_samples_per_pixel
    # every camera ray, once (pixel-major, spp samples per pixel)
    rays = []
    for k in range(len(w.cameras)):
        ys, xs = np.mgrid[0:H, 0:W]
        px, py = np.repeat(xs.reshape(-1), spp), np.repeat(ys.reshape(-1), spp)
        sm = np.tile(np.arange(spp), W * H)
        rays.append(O.camera_rays(O.camera16(w.cameras[k], W, H), W, spp, cfg.seed, px, py, sm))
    p0 = E.params_from(g)
    em = torch.tensor(w.emission, dtype=torch.float64)
    env1 = torch.tensor(w.env_constant, dtype=torch.float64)
    rng = np.random.default_rng(11)
    ls_np = np.asarray(g.scale, np.float64)

    def affected(i):
        lo, hi = E.box_3sigma(g.mean[i], ls_np[i], g.quat_wxyz[i], pad=0.05)
        return [np.unique(np.nonzero(E.slab_hits(o.astype(np.float64), d.astype(np.float64), lo, hi))[0] // spp)
                for o, d in rays]

    # 8 random Gaussians that at least 100 pixels see; their 11 geometry parameters each (mean 3,
    # log-scale 3, quaternion 4, density 1); the first 64 that finite differences resolve
    chosen = []
    for i in rng.permutation(n):
        pix = affected(int(i))
        if sum(len(a) for a in pix) >= 100:
            chosen.append((int(i), pix))
        if len(chosen) == 8:
            break
    # The loss differentiated is the FP64 one: on every pixel a chosen Gaussian touches, the
    # adjoint's upstream gradient is 2 (L64 - target) with L64 from the oracle (elsewhere the
    # GPU image's; those pixels do not reach the chosen Gaussians).  The forward's own error is
    # gated by test_forward_matches_fp64.
    dls = []
    for k in range(len(w.cameras)):
        dl = np.zeros((H, W, 4), np.float32)
        dl[..., :3] = 2.0 * (c5["imgs"][k] - c5["targets"][k])
        union = np.unique(np.concatenate([p[k] for _, p in chosen]))
        if len(union):
            rows = (union[:, None] * spp + np.arange(spp)[None, :]).reshape(-1)
            S, C = c5["osc"].emission_sums(w.emission, rays[k][0][rows], rays[k][1][rows])
            L = E.radiance(torch.tensor(S), torch.tensor(C), env1.expand(len(rows), 3)).numpy()
            pix64 = L.reshape(len(union), spp, 3).mean(1)
            dl.reshape(-1, 4)[union, :3] = 2.0 * (pix64 - c5["targets"][k].reshape(-1, 3)[union])
        dls.append(dl)
    grads_by = {}
    for prec in ("fast", "accurate"):
        pcfg = vp.Config(**{**cfg.__dict__, "precision": prec})
        grads_by[prec] = zero_grads(n)
        for k, cam in enumerate(w.cameras):
            render_emission_backward(c5["scene"], c5["env"], cam, pcfg, dls[k], grads_by[prec])
    results = []
    for i, pix_sets in chosen:
        # per camera: FP64 sums of every other Gaussian on the affected pixels' rays (fixed)
        parts = []
        for k, pixels in enumerate(pix_sets):
            if len(pixels) == 0:
                continue
            rows = (pixels[:, None] * spp + np.arange(spp)[None, :]).reshape(-1)
            o, d = rays[k][0][rows], rays[k][1][rows]
            S, C = c5["osc"].emission_sums(w.emission, o, d, exclude=i)
            tgt = torch.tensor(c5["targets"][k].reshape(-1, 3)[pixels])
            parts.append((torch.tensor(o, dtype=torch.float64), torch.tensor(d, dtype=torch.float64),
                          torch.tensor(S), torch.tensor(C), tgt, len(pixels)))

        allo = torch.cat([p[0] for p in parts])
        alld = torch.cat([p[1] for p in parts])
        ri_all = torch.arange(len(allo))
        gi_all = torch.full((len(allo),), i, dtype=torch.int64)

        def pixels_with(pp):
            out = []
            for ot, dt, S, C, tgt, npx in parts:
                ri = torch.arange(len(ot))
                gi = torch.full((len(ot),), i, dtype=torch.int64)
                tau, valid = E.pair_tau(pp, w.sigma_multiplier, ot, dt, ri, gi)
                ti = torch.zeros(len(ot), dtype=torch.float64)
                ti[valid] = tau
                L = E.radiance(S + ti, C + ti[:, None] * em[i], env1.expand(len(ot), 3))
                out.append(L.reshape(npx, spp, 3).mean(1))
            return out

        for key, gkey, comps in (("mean", "mean", 3), ("log_scale", "scale", 3), ("quat", "quat_wxyz", 4),
                                 ("density", "density", 1)):
            for c in range(comps):
                idx = (i, c) if comps > 1 else (i,)
                scale = max(1.0, abs(float(p0[key][idx])))
                # step: well inside the parameter distance at which any ray's d2 first reaches 9
                # (the 3-sigma kink, where tau ~ sqrt(9 - d2) has no Taylor expansion)
                delta = 1e-8 * scale
                d2 = []
                for sgn in (1, 0, -1):
                    pp = {kk: v.clone() for kk, v in p0.items()}
                    pp[key][idx] += sgn * delta
                    d2.append(E.pair_d2(pp, allo, alld, ri_all, gi_all))
                slope = (d2[0] - d2[2]).abs() / (2 * delta)
                near = (d2[1] - 9.0).abs() < 0.5
                kink = float(((d2[1] - 9.0).abs()[near] / slope[near].clamp(min=1e-300)).min()) if near.any() else 1.0
                eps = min(1e-6 * scale, 0.02 * kink)
                if eps < 1e-9 * scale:
                    continue  # a ray grazes the 3-sigma surface within 5e-8: no finite difference resolves it
                Lp, Lm = [], []
                for sgn, dst in ((1, Lp), (-1, Lm)):
                    pp = {kk: v.clone() for kk, v in p0.items()}
                    pp[key][idx] += sgn * eps
                    dst.extend(pixels_with(pp))
                # Loss(+) - Loss(-) = sum (L+ - L-)(L+ + L- - 2 t), without the large common part
                diff = sum(float(((a - b) * (a + b - 2.0 * part[4])).sum()) for a, b, part in zip(Lp, Lm, parts))
                fd = diff / (2 * eps)
                got = {prec: float(gr[gkey][i * comps + c]) for prec, gr in grads_by.items()}
                results.append((key, i, c, fd, got))
    results = results[:64]
    assert len(results) == 64
    G = max(abs(r[3]) for r in results)
    assert G > 0
    for prec in grads_by:
        bad = [(r[0], r[1], r[2], r[3], r[4][prec]) for r in results
               if not abs(r[4][prec] - r[3]) <= 1e-3 * abs(r[3]) + 1e-6 * G]
        assert not bad, (prec, bad)


def test_autograd_function_matches_the_adjoint(c5, vp_ctx):
    from volprim_b200.autograd import render_emission_images
    w = c5["w"]
    g = w.gaussians
    dev = torch.device("cuda", 0)
    t = {k: torch.tensor(np.asarray(v, np.float32), device=dev, requires_grad=True)
         for k, v in (("mean", g.mean), ("ls", g.scale), ("q", g.quat_wxyz), ("dens", g.density), ("em", w.emission))}
    imgs = render_emission_images(t["mean"], t["ls"], t["q"], t["dens"], t["em"], w.cameras[:2], w.config, c5["env"],
                                  w.sigma_multiplier, vp_ctx)
    for k in range(2):  # the scene rebuilt from the tensors renders the same image
        a = imgs[k].detach().cpu().numpy().astype(np.float64)
        assert np.allclose(a, c5["imgs"][k], rtol=1e-6, atol=1e-7)
    target = torch.tensor(np.stack(c5["targets"][:2]), dtype=torch.float32, device=dev)
    loss = ((imgs - target) ** 2).sum()
    loss.backward()
    ref = zero_grads(g.count)
    for k in range(2):
        dl = np.zeros((w.config.image_height, w.config.image_width, 4), np.float32)
        dl[..., :3] = 2.0 * (c5["imgs"][k] - c5["targets"][k])
        render_emission_backward(c5["scene"], c5["env"], w.cameras[k], w.config, dl, ref)
    for key, tk in (("mean", "mean"), ("scale", "ls"), ("quat_wxyz", "q"), ("density", "dens"), ("emission", "em")):
        a = t[tk].grad.detach().cpu().numpy().reshape(-1).astype(np.float64)
        b = ref[key].astype(np.float64)
        assert np.linalg.norm(a - b) <= 1e-4 * np.linalg.norm(b), key  # same kernels, atomic order aside
    # a small step against the gradient lowers the loss
    with torch.no_grad():
        step = {k: v - 1e-4 * v.grad / (v.grad.norm() + 1e-30) * v.norm() for k, v in t.items()}
    imgs2 = render_emission_images(step["mean"], step["ls"], step["q"], step["dens"], step["em"], w.cameras[:2],
                                   w.config, c5["env"], w.sigma_multiplier, vp_ctx)
    assert float(((imgs2 - target) ** 2).sum().detach()) < float(loss.detach())


def test_adjoint_with_many_hits_per_ray(vp_ctx):
    """A stack of 150 overlapping Gaussians along the view axis: central rays cross all of them
    (well over the 64-hit regime of the differentiation workload), edge rays few or none.  The
    adjoint must match FP64 autodiff of the same closed form with the crop test's tolerances."""
    rng = np.random.default_rng(21)
    n = 150
    mean = np.stack([rng.normal(0, 0.02, n), rng.normal(0, 0.02, n), np.linspace(-1.5, 1.5, n)], 1).astype(np.float32)
    log_scale = rng.normal(np.log(0.12), 0.2, (n, 3)).astype(np.float32)
    g = vp.Gaussians(mean, log_scale, scenes.uniform_quaternions(rng, n), np.exp(rng.normal(-5.0, 0.3, n)).astype(np.float32),
                     None, scale_is_log=True)
    emission = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    res, spp = 24, 2
    cam = vp.Camera.perspective((0.0, 0.0, -3.5), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 40.0)
    env_c = (0.3, 0.4, 0.5)
    sc = vp.Scene(vp_ctx, g, 1.0)
    sc.set_emission(emission)
    env = vp.Environment(vp_ctx, constant=env_c)
    cfg = vp.Config(num_samples_per_pixel=spp, image_width=res, image_height=res, seed=3, precision="fast")
    ys, xs = np.mgrid[0:res, 0:res]
    px, py = np.repeat(xs.reshape(-1), spp), np.repeat(ys.reshape(-1), spp)
    sm = np.tile(np.arange(spp), res * res)
    o, d = O.camera_rays(O.camera16(cam, res, res), res, spp, cfg.seed, px, py, sm)
    osc = O.OracleScene.from_gaussians(g, 1.0)
    ri, gi = osc.ray_candidates(o, d)
    p = E.params_from(g, requires_grad=True)
    _, valid = E.pair_tau(p, 1.0, torch.tensor(o, dtype=torch.float64), torch.tensor(d, dtype=torch.float64),
                          torch.tensor(ri), torch.tensor(gi))
    hits = np.bincount(ri[valid.numpy()], minlength=len(o))
    assert (hits > 64).sum() >= 32 and (hits < 64).sum() >= 32, (hits.min(), hits.max())
    em = torch.tensor(emission, dtype=torch.float64, requires_grad=True)
    S, C = E.ray_sums(p, em, 1.0, torch.tensor(o, dtype=torch.float64), torch.tensor(d, dtype=torch.float64),
                      torch.tensor(ri), torch.tensor(gi), len(o))
    L = E.radiance(S, C, torch.tensor(env_c, dtype=torch.float64).expand(len(o), 3))
    pix = L.reshape(res * res, spp, 3).mean(1).reshape(res, res, 3)
    up = torch.tensor(rng.normal(0, 1, (res, res, 3)))
    (pix * up).sum().backward()
    dl = np.zeros((res, res, 4), np.float32)
    dl[..., :3] = up.numpy()
    ref = {"mean": p["mean"].grad.numpy().reshape(-1), "scale": p["log_scale"].grad.numpy().reshape(-1),
           "quat_wxyz": p["quat"].grad.numpy().reshape(-1), "density": p["density"].grad.numpy().reshape(-1),
           "emission": em.grad.numpy().reshape(-1)}
    for prec in ("fast", "accurate"):
        c = vp.Config(**{**cfg.__dict__, "precision": prec})
        got_g = zero_grads(n)
        render_emission_backward(sc, env, cam, c, dl, got_g)
        for key, r in ref.items():
            got = got_g[key].astype(np.float64)
            rel = np.linalg.norm(got - r) / np.linalg.norm(r)
            assert rel <= 1e-3, (prec, key, rel)
            big = np.abs(r) > 1e-2 * np.abs(r).max()
            assert np.all(np.abs(got[big] - r[big]) <= 1e-2 * np.abs(r[big])), (prec, key)
    env.close()
    sc.close()
