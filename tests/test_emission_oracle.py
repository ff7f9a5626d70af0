"""CPU: the FP64 PyTorch restatement of the absorption-plus-emission model (oracle/emission_oracle.py)
against the C++ FP64 closed-form transmittance oracle (which the reference pins), its closed
forms in the limits where the model is exact, and its autograd gradients against central
finite differences of itself."""
import math

import numpy as np
import torch

import oracle as O
import emission_oracle as E
import volprim_b200 as vp
from volprim_b200 import scenes


def small_scene(seed=0, n=60):
    rng = np.random.default_rng(seed)
    mean = rng.uniform(-0.5, 0.5, (n, 3)).astype(np.float32)
    ls = rng.normal(math.log(0.15), 0.3, (n, 3)).astype(np.float32)
    q = scenes.uniform_quaternions(rng, n) * rng.uniform(0.5, 2.0, (n, 1)).astype(np.float32)  # unnormalised
    dens = np.exp(rng.normal(0.0, 0.5, n)).astype(np.float32)
    return vp.Gaussians(mean, ls, q, dens, None, scale_is_log=True)


def rays(seed, n):
    rng = np.random.default_rng(seed)
    o = rng.normal(size=(n, 3))
    o = 2.5 * o / np.linalg.norm(o, axis=1, keepdims=True)
    o[: n // 4] = rng.uniform(-0.3, 0.3, (n // 4, 3))  # a quarter start inside the cloud
    d = rng.uniform(-0.4, 0.4, (n, 3)) - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return o.astype(np.float32), d.astype(np.float32)


def test_tau_matches_cpp_fp64_closed_form():
    g = small_scene()
    osc = O.OracleScene.from_gaussians(g, sigma_multiplier=1.7, use_bvh=True)
    o, d = rays(1, 400)
    _, tau_ref = osc.transmittance_fp64(o, d)
    ri, gi = osc.ray_candidates(o, d)
    p = E.params_from(g)
    S, _ = E.ray_sums(p, torch.zeros((g.count, 3), dtype=torch.float64), 1.7, torch.tensor(o, dtype=torch.float64),
                      torch.tensor(d, dtype=torch.float64), torch.tensor(ri), torch.tensor(gi), len(o))
    assert (tau_ref > 0.1).sum() > 100
    # the C++ oracle rounds exp(log-scale) and the normalised quaternion to FP32 as the reference's
    # Primitive constructor does (primitive.h:80-87, quat.h:55-58); the restatement stays FP64
    assert np.allclose(S.numpy(), tau_ref, rtol=2e-6, atol=1e-12)


def test_candidates_cover_all_contributing_pairs():
    g = small_scene(2)
    osc = O.OracleScene.from_gaussians(g, use_bvh=True)
    o, d = rays(3, 200)
    ri, gi = osc.ray_candidates(o, d)
    all_ri = np.repeat(np.arange(len(o)), g.count)
    all_gi = np.tile(np.arange(g.count), len(o))
    p = E.params_from(g)
    args = (torch.tensor(o, dtype=torch.float64), torch.tensor(d, dtype=torch.float64))
    _, v_all = E.pair_tau(p, 1.0, *args, torch.tensor(all_ri), torch.tensor(all_gi))
    _, v_c = E.pair_tau(p, 1.0, *args, torch.tensor(ri), torch.tensor(gi))
    assert int(v_all.sum()) == int(v_c.sum()) > 0


def test_single_gaussian_emission_is_exact():
    # one Gaussian: L = e (1 - T) + T env exactly (int sigma e T dt = e (1 - T))
    g = vp.Gaussians(np.zeros((1, 3), np.float32), np.full((1, 3), math.log(0.3), np.float32),
                     np.array([[1.0, 0.0, 0.0, 0.0]], np.float32), np.array([2.0], np.float32), None, scale_is_log=True)
    p = E.params_from(g)
    e = torch.tensor([[0.2, 0.5, 0.9]], dtype=torch.float64)
    o = torch.tensor([[0.0, 0.1, -3.0]], dtype=torch.float64)
    d = torch.tensor([[0.0, 0.0, 1.0]], dtype=torch.float64)
    S, C = E.ray_sums(p, e, 1.0, o, d, torch.tensor([0]), torch.tensor([0]), 1)
    env = torch.tensor([[1.0, 0.7, 0.3]], dtype=torch.float64)
    L = E.radiance(S, C, env)
    T = math.exp(-float(S[0]))
    want = e[0] * (1 - T) + T * env[0]
    assert torch.allclose(L[0], want, rtol=1e-14, atol=0)
    # closed form of the chord through an isotropic Gaussian at distance 0.1 from its centre
    s = math.exp(float(np.float32(math.log(0.3))))  # the float32 log-scale the Gaussian holds
    dperp = 0.1 / s
    tau = 2.0 / (2 * math.pi * s * s) * math.exp(-0.5 * dperp ** 2) * math.erf(math.sqrt((9 - dperp ** 2) / 2))
    assert abs(float(S[0]) - tau) < 1e-12 * tau


def test_autograd_matches_central_differences():
    g = small_scene(4, n=30)
    osc = O.OracleScene.from_gaussians(g, use_bvh=True)
    o, d = rays(5, 120)
    ri, gi = (torch.tensor(a) for a in osc.ray_candidates(o, d))
    ot, dt = torch.tensor(o, dtype=torch.float64), torch.tensor(d, dtype=torch.float64)
    rng = np.random.default_rng(6)
    em = torch.tensor(rng.uniform(0, 1, (g.count, 3)), dtype=torch.float64, requires_grad=True)
    env = torch.ones((len(o), 3), dtype=torch.float64) * 0.5
    target = torch.tensor(rng.uniform(0, 1, (len(o), 3)), dtype=torch.float64)

    def loss(p, e):
        S, C = E.ray_sums(p, e, 1.3, ot, dt, ri, gi, len(o))
        return ((E.radiance(S, C, env) - target) ** 2).sum()

    p = E.params_from(g, requires_grad=True)
    loss(p, em).backward()
    checked = 0
    for key, comps in (("mean", 3), ("log_scale", 3), ("quat", 4), ("density", 1)):
        for i in rng.choice(g.count, 4, replace=False):
            for c in range(comps):
                idx = (i, c) if comps > 1 else (i,)
                eps = 1e-6 * max(1.0, abs(float(p[key].detach()[idx])))
                vals = []
                for sgn in (1, -1):
                    q = {k: v.detach().clone() for k, v in p.items()}
                    q[key][idx] += sgn * eps
                    vals.append(float(loss(q, em.detach())))
                fd = (vals[0] - vals[1]) / (2 * eps)
                ad = float(p[key].grad[idx])
                assert abs(fd - ad) <= 1e-5 * max(abs(fd), 1e-3), (key, i, c, fd, ad)
                checked += 1
    assert checked == 4 * 11


def test_cpp_emission_sums_match_the_restatement():
    g = small_scene(7)
    osc = O.OracleScene.from_gaussians(g, sigma_multiplier=1.2, use_bvh=True)
    o, d = rays(8, 300)
    em = np.random.default_rng(9).uniform(0, 1, (g.count, 3)).astype(np.float32)
    S_c, C_c = osc.emission_sums(em, o, d)
    ri, gi = osc.ray_candidates(o, d)
    S, C = E.ray_sums(E.params_from(g), torch.tensor(em, dtype=torch.float64), 1.2, torch.tensor(o, dtype=torch.float64),
                      torch.tensor(d, dtype=torch.float64), torch.tensor(ri), torch.tensor(gi), len(o))
    assert np.allclose(S_c, S.numpy(), rtol=2e-6, atol=1e-12)
    assert np.allclose(C_c, C.numpy(), rtol=2e-6, atol=1e-12)
    # excluding one Gaussian removes exactly its share
    S_x, _ = osc.emission_sums(em, o, d, exclude=5)
    keep = gi != 5
    S5, _ = E.ray_sums(E.params_from(g), torch.tensor(em, dtype=torch.float64), 1.2, torch.tensor(o, dtype=torch.float64),
                       torch.tensor(d, dtype=torch.float64), torch.tensor(ri[keep]), torch.tensor(gi[keep]), len(o))
    assert np.allclose(S_x, S5.numpy(), rtol=2e-6, atol=1e-12)
    assert (S_c - S_x).max() > 0
