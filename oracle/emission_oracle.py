"""ORACLE — test infrastructure only (tests/ and bench.py's CPU-baseline leg; never the product).

FP64 restatement of the absorption-plus-emission image model that vp_render_emission computes,
in PyTorch float64 on the CPU so that autograd gives the reference gradients:

  per (ray, Gaussian) pair: the closed-form optical depth of the 3-sigma chord over [0, inf)
  (Primitive::optical_depth, primitive.h:249-318, with t0 = max(t_entry, 0) and the
  RAY_SEGMENT_MIN_LENGTH rule), through the whitening W = diag(1/s) R(q/|q|)^T of the caller's
  parameters (mean, log-scale, quaternion (w,x,y,z), density x sigma-multiplier);
  per ray: S = sum tau, C = sum tau e, L = (1 - exp(-S)) C / S + exp(-S) env(d).

Candidate (ray, Gaussian) pairs come from the C++ oracle's CPU BVH (OracleScene.ray_candidates);
pairs whose chord misses are dropped before the differentiable evaluation.
"""
from __future__ import annotations

import math

import numpy as np
import torch

SQRT_HALF_PI = math.sqrt(math.pi / 2.0)
INV_TWO_PI_POW_1_5 = (2.0 * math.pi) ** -1.5
SEGMENT_MIN = 1e-6


def rotation(q):
    """R(q / |q|) for (P, 4) quaternions (w, x, y, z): rows as the build's forward rotation."""
    q = q / q.norm(dim=1, keepdim=True)
    w, x, y, z = q.unbind(1)
    return torch.stack([
        torch.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)], 1),
        torch.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)], 1),
        torch.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], 1)], 1)


def pair_tau(params, sigma_multiplier, o, d, ri, gi):
    """tau of each (ray ri, Gaussian gi) pair and the mask of pairs that contribute.

    params: dict of float64 tensors mean (N,3), log_scale (N,3), quat (N,4), density (N,);
    o, d: (R, 3) float64 tensors; ri, gi: int64 tensors.  Returns (tau[valid pairs], valid)."""
    def geometry(mean, log_scale, quat):
        R = rotation(quat[gi])
        s = torch.exp(log_scale[gi])
        v = o[ri] - mean[gi]
        p = torch.einsum("plk,pl->pk", R, v) / s
        w = torch.einsum("plk,pl->pk", R, d[ri]) / s
        A = (w * w).sum(1)
        B = (p * w).sum(1)
        d2 = (p * p).sum(1) - B * B / A
        return s, A, B, d2

    with torch.no_grad():
        _, A, B, d2 = geometry(params["mean"], params["log_scale"], params["quat"])
        h = torch.sqrt(torch.clamp(9.0 - d2, min=0.0))
        sA = torch.sqrt(A)
        tc = -B / A
        t_in, t_out = tc - h / sA, tc + h / sA
        valid = (d2 < 9.0) & (t_out > 0) & (t_out - torch.clamp(t_in, min=0.0) > SEGMENT_MIN)
        inside = t_in < 0
    ri_v, gi_v = ri[valid], gi[valid]
    sub = {k: v for k, v in params.items()}
    R = rotation(sub["quat"][gi_v])
    s = torch.exp(sub["log_scale"][gi_v])
    v = o[ri_v] - sub["mean"][gi_v]
    p = torch.einsum("plk,pl->pk", R, v) / s
    w = torch.einsum("plk,pl->pk", R, d[ri_v]) / s
    A = (w * w).sum(1)
    B = (p * w).sum(1)
    d2 = (p * p).sum(1) - B * B / A
    h = torch.sqrt(9.0 - d2)
    sA = torch.sqrt(A)
    u = torch.where(inside[valid], B / sA, -h)
    icf = sub["density"][gi_v] * sigma_multiplier * INV_TWO_PI_POW_1_5 / s.prod(1) * SQRT_HALF_PI
    tau = icf / sA * torch.exp(-0.5 * d2) * (torch.erf(h / math.sqrt(2.0)) - torch.erf(u / math.sqrt(2.0)))
    return tau, valid


def pair_d2(params, o, d, ri, gi):
    """Squared whitened distance of closest approach of each (ray, Gaussian) pair: the chord
    exists where d2 < 9, and tau has a square-root kink at d2 = 9 (the 3-sigma truncation)."""
    R = rotation(params["quat"][gi])
    s = torch.exp(params["log_scale"][gi])
    p = torch.einsum("plk,pl->pk", R, o[ri] - params["mean"][gi]) / s
    w = torch.einsum("plk,pl->pk", R, d[ri]) / s
    B = (p * w).sum(1)
    return (p * p).sum(1) - B * B / (w * w).sum(1)


def ray_sums(params, emission, sigma_multiplier, o, d, ri, gi, n_rays):
    """(S (R,), C (R, 3)) per ray."""
    tau, valid = pair_tau(params, sigma_multiplier, o, d, ri, gi)
    ri_v, gi_v = ri[valid], gi[valid]
    S = torch.zeros(n_rays, dtype=torch.float64).index_add(0, ri_v, tau)
    C = torch.zeros((n_rays, 3), dtype=torch.float64).index_add(0, ri_v, tau[:, None] * emission[gi_v])
    return S, C


def radiance(S, C, env):
    """L = (1 - T) C / S + T env, T = exp(-S) (env where S = 0)."""
    T = torch.exp(-S)
    safe = torch.where(S > 1e-12, S, torch.ones_like(S))
    a = torch.where(S > 1e-12, -torch.expm1(-safe) / safe, 1.0 - 0.5 * S)
    return a[:, None] * C + T[:, None] * env


def params_from(g, dtype=torch.float64, requires_grad=False):
    """float64 tensors of a Gaussians record whose scales are logs (scale_is_log=True)."""
    assert g.scale_is_log
    out = {"mean": torch.tensor(np.asarray(g.mean, np.float64).reshape(-1, 3), dtype=dtype),
           "log_scale": torch.tensor(np.asarray(g.scale, np.float64).reshape(-1, 3), dtype=dtype),
           "quat": torch.tensor(np.asarray(g.quat_wxyz, np.float64).reshape(-1, 4), dtype=dtype),
           "density": torch.tensor(np.asarray(g.density, np.float64).reshape(-1), dtype=dtype)}
    for v in out.values():
        v.requires_grad_(requires_grad)
    return out


def slab_hits(o, d, lo, hi):
    """Rays (numpy (R,3)) over [0, inf) that meet the box [lo, hi]."""
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = 1.0 / np.where(np.abs(d) < 1e-300, 1e-300, d)
        t0 = (lo[None, :] - o) * inv
        t1 = (hi[None, :] - o) * inv
    tn = np.maximum(np.minimum(t0, t1).max(1), 0.0)
    tf = np.maximum(t0, t1).min(1)
    return tn <= tf


def box_3sigma(mean, log_scale, quat, pad=0.05):
    """World box of a Gaussian's 3-sigma ellipsoid, inflated by `pad` (relative)."""
    R = rotation(torch.tensor(np.asarray(quat, np.float64)[None, :]))[0].numpy()
    s = np.exp(np.asarray(log_scale, np.float64))
    e = 3.0 * np.sqrt(((R * s[None, :]) ** 2).sum(1)) * (1.0 + pad)
    m = np.asarray(mean, np.float64)
    return m - e, m + e
