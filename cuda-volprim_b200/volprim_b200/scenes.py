"""Seeded synthetic workloads: Gaussian mixtures, procedural HDR environment, cameras.

No dataset or asset ships with the reference for these workloads (its PLY assets and HDR maps
are absent), so every scene here is generated from a seed with the stated distributions:
  absorption_256     256 Gaussians, means U[-1,1]^3, scales logN(ln 0.1, 0.4), uniform
                     quaternions, densities logN(ln 5, 0.5), albedo 0; constant white env;
                     pinhole at distance 3.5 (eye (0,0,-3.5) looking at the origin, the
                     reference's asset_validation "negz" view, test/scenes/cloud_validation.cpp:
                     114-129), vfov 40 deg, 128x128, 16 spp, seed 0.
  showcase_500k      means by thresholding a seeded 3-D value-noise field in [-1,1]x[-1/2,1/2]^2,
                     scales logN(ln 0.02, 0.5), densities logN(0, 0.7) x sigma-multiplier 7.5,
                     albedo 0.9, isotropic phase, procedural 2048x1024 environment, MIS NEE,
                     RR from depth 12, max depth 64, 512x512, 256 spp.
  stress_2m          2M Gaussians around 16 isotropic normal clusters (std 0.15), scales
                     logN(ln 0.05, 0.3), densities logN(ln 2, 0.5), albedo 0.8, same env,
                     1024x1024, 64 spp.
  serving_4          the serving form's resident scenes: showcase_500k's generator at 50k, 100k,
                     250k and 500k Gaussians with seeds 1-4 (sigma-multiplier 7.5), each with the
                     procedural environment; requests from volprim_b200.serving.make_trace.
  emission_100k      the differentiation form: 100k Gaussians with showcase_500k's distributions
                     (log-scales as the parameters), RGB emission U[0,1], sigma-multiplier 7.5,
                     4 cameras at distance 3.5 in seeded directions looking at the origin,
                     256x256, 8 spp, constant white environment.
Densities are the reference's mass convention (ply.cpp:107-116).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .api import Camera, Config, Gaussians


def uniform_quaternions(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniform rotations (Shoemake 1992), returned as (w, x, y, z)."""
    u1, u2, u3 = rng.random((3, n))
    a, b = np.sqrt(1.0 - u1), np.sqrt(u1)
    x = a * np.sin(2 * np.pi * u2)
    y = a * np.cos(2 * np.pi * u2)
    z = b * np.sin(2 * np.pi * u3)
    w = b * np.cos(2 * np.pi * u3)
    return np.stack([w, x, y, z], axis=1).astype(np.float32)


def _lognormal(rng, mu, sigma, shape):
    return np.exp(rng.normal(mu, sigma, shape)).astype(np.float32)


@dataclass
class Workload:
    name: str
    gaussians: Gaussians
    sigma_multiplier: float
    camera: Camera
    config: Config
    env: object  # None = constant white, else (H, W, 3) float32

    @property
    def paths(self) -> int:
        c = self.config
        return c.image_width * c.image_height * c.num_samples_per_pixel


def absorption_gaussians(n: int = 256, seed: int = 0) -> Gaussians:
    rng = np.random.default_rng(seed)
    mean = rng.uniform(-1.0, 1.0, (n, 3)).astype(np.float32)
    scale = _lognormal(rng, math.log(0.1), 0.4, (n, 3))
    quat = uniform_quaternions(rng, n)
    density = _lognormal(rng, math.log(5.0), 0.5, (n,))
    albedo = np.zeros((n, 3), np.float32)
    return Gaussians(mean, scale, quat, density, albedo)


def value_noise(points: np.ndarray, seed: int, cells=(8, 4, 4), octaves: int = 3,
                lo=(-1.0, -0.5, -0.5), hi=(1.0, 0.5, 0.5)) -> np.ndarray:
    """Seeded 3-D value noise (smoothstep-trilinear lattice noise, octaves halving in amplitude)."""
    rng = np.random.default_rng(seed)
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    u = (points - lo) / (hi - lo)
    total = np.zeros(points.shape[0])
    amp, norm = 1.0, 0.0
    for o in range(octaves):
        c = np.asarray(cells) * (2 ** o)
        lat = rng.random((c[0] + 1, c[1] + 1, c[2] + 1))
        x = np.clip(u, 0.0, 1.0) * c
        i = np.minimum(np.floor(x).astype(np.int64), c - 1)
        f = x - i
        f = f * f * (3.0 - 2.0 * f)
        acc = np.zeros(points.shape[0])
        for dx in (0, 1):
            wx = f[:, 0] if dx else 1.0 - f[:, 0]
            for dy in (0, 1):
                wy = f[:, 1] if dy else 1.0 - f[:, 1]
                for dz in (0, 1):
                    wz = f[:, 2] if dz else 1.0 - f[:, 2]
                    acc += wx * wy * wz * lat[i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz]
        total += amp * acc
        norm += amp
        amp *= 0.5
    return total / norm


def showcase_gaussians(n: int = 500_000, seed: int = 0, threshold: float = 0.55) -> Gaussians:
    """Means where the value noise exceeds `threshold` inside the 2x1x1 box (rejection sampling)."""
    rng = np.random.default_rng(seed)
    lo = np.array([-1.0, -0.5, -0.5])
    hi = np.array([1.0, 0.5, 0.5])
    kept = []
    have = 0
    while have < n:
        cand = lo + (hi - lo) * rng.random((max(4 * (n - have), 4096), 3))
        keep = cand[value_noise(cand, seed + 7919) > threshold]
        kept.append(keep)
        have += keep.shape[0]
    mean = np.concatenate(kept)[:n].astype(np.float32)
    scale = _lognormal(rng, math.log(0.02), 0.5, (n, 3))
    quat = uniform_quaternions(rng, n)
    density = _lognormal(rng, 0.0, 0.7, (n,))
    albedo = np.full((n, 3), 0.9, np.float32)
    return Gaussians(mean, scale, quat, density, albedo)


def stress_gaussians(n: int = 2_000_000, seed: int = 0, clusters: int = 16) -> Gaussians:
    rng = np.random.default_rng(seed)
    centers = rng.uniform(-0.7, 0.7, (clusters, 3))
    which = rng.integers(0, clusters, n)
    mean = (centers[which] + rng.normal(0.0, 0.15, (n, 3))).astype(np.float32)
    scale = _lognormal(rng, math.log(0.05), 0.3, (n, 3))
    quat = uniform_quaternions(rng, n)
    density = _lognormal(rng, math.log(2.0), 0.5, (n,))
    albedo = np.full((n, 3), 0.8, np.float32)
    return Gaussians(mean, scale, quat, density, albedo)


def procedural_env(width: int = 2048, height: int = 1024, sun_dir=(0.7197, 0.4530, 0.5261),
                   sun_radiance: float = 1e4, sun_radius_deg: float = 0.5) -> np.ndarray:
    """Lat-long HDR (rows = polar angle from +y, u = atan2(z, x)/2pi + 1/2, as the reference's
    lookup): sky gradient above the horizon, dim ground below, and a sun disc of radiance
    `sun_radiance` relative to the sky over `sun_radius_deg` degrees."""
    v = (np.arange(height) + 0.5) / height
    u = (np.arange(width) + 0.5) / width
    polar = v * np.pi
    theta = (u - 0.5) * 2.0 * np.pi
    sp, cp = np.sin(polar)[:, None], np.cos(polar)[:, None]
    dx = sp * np.cos(theta)[None, :]
    dy = np.broadcast_to(cp, (height, width))
    dz = sp * np.sin(theta)[None, :]
    up = np.clip(dy, 0.0, 1.0)
    sky = np.stack([0.35 + 0.25 * (1 - up), 0.55 + 0.25 * (1 - up), 0.95 - 0.1 * up], axis=-1)
    ground = np.broadcast_to(np.array([0.08, 0.07, 0.06]), sky.shape)
    img = np.where((dy >= 0.0)[..., None], sky, ground)
    s = np.asarray(sun_dir, np.float64)
    s = s / np.linalg.norm(s)
    cosang = dx * s[0] + dy * s[1] + dz * s[2]
    sun = cosang >= math.cos(math.radians(sun_radius_deg))
    img = img.copy()
    img[sun] = np.array([1.0, 0.95, 0.85]) * sun_radiance
    return np.ascontiguousarray(img, dtype=np.float32)


def negz_camera(distance: float = 3.5, vfov: float = 40.0) -> Camera:
    return Camera.perspective((0.0, 0.0, -distance), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), vfov)


def absorption_256(seed: int = 0, res: int = 128, spp: int = 16) -> Workload:
    cfg = Config(num_samples_per_pixel=spp, image_width=res, image_height=res, seed=seed, hg_g=0.0)
    return Workload("absorption_256", absorption_gaussians(256, seed), 1.0, negz_camera(), cfg, None)


def showcase_500k(seed: int = 0, n: int = 500_000, res: int = 512, spp: int = 256,
                  env_size=(2048, 1024)) -> Workload:
    cfg = Config(num_samples_per_pixel=spp, image_width=res, image_height=res, seed=seed, hg_g=0.0,
                 max_bounces=64, rr_depth=12, nee="mis")
    env = procedural_env(*env_size)
    return Workload("showcase_500k", showcase_gaussians(n, seed), 7.5, negz_camera(), cfg, env)


def stress_2m(seed: int = 0, n: int = 2_000_000, res: int = 1024, spp: int = 64,
              env_size=(2048, 1024)) -> Workload:
    cfg = Config(num_samples_per_pixel=spp, image_width=res, image_height=res, seed=seed, hg_g=0.0,
                 max_bounces=64, rr_depth=12, nee="mis")
    env = procedural_env(*env_size)
    return Workload("stress_2m", stress_gaussians(n, seed), 1.0, negz_camera(), cfg, env)


@dataclass
class EmissionWorkload:
    name: str
    gaussians: Gaussians     # scale_is_log=True: the log-scales are the differentiated parameters
    emission: np.ndarray     # (N, 3) RGB per unit optical depth
    sigma_multiplier: float
    cameras: list
    config: Config
    env_constant: tuple      # constant environment radiance (RGB)


def sphere_cameras(rng: np.random.Generator, k: int, distance: float = 3.5, vfov: float = 40.0) -> list:
    """k pinhole cameras at `distance` from the origin in uniform random directions, looking at it."""
    cams = []
    for _ in range(k):
        v = rng.normal(size=3)
        v /= np.linalg.norm(v)
        up = (0.0, 1.0, 0.0) if abs(v[1]) < 0.95 else (0.0, 0.0, 1.0)
        cams.append(Camera.perspective(tuple(float(x) for x in distance * v), (0.0, 0.0, 0.0), up, vfov))
    return cams


def emission_100k(seed: int = 0, n: int = 100_000, res: int = 256, spp: int = 8, n_cams: int = 4) -> EmissionWorkload:
    g = showcase_gaussians(n, seed)
    rng = np.random.default_rng(seed + 101)
    emission = rng.uniform(0.0, 1.0, (n, 3)).astype(np.float32)
    gl = Gaussians(g.mean, np.log(g.scale).astype(np.float32), g.quat_wxyz, g.density, None, scale_is_log=True)
    cfg = Config(num_samples_per_pixel=spp, image_width=res, image_height=res, seed=seed, precision="fast")
    return EmissionWorkload("emission_100k", gl, emission, 7.5, sphere_cameras(rng, n_cams), cfg, (1.0, 1.0, 1.0))


def perturbed(w: EmissionWorkload, seed: int = 1) -> tuple:
    """Seeded perturbation of a workload's parameters (the target of the image loss):
    (Gaussians, emission)."""
    rng = np.random.default_rng(seed)
    g = w.gaussians
    n = g.count
    mean = (g.mean + rng.normal(0.0, 0.005, (n, 3))).astype(np.float32)
    ls = (g.scale + rng.normal(0.0, 0.05, (n, 3))).astype(np.float32)
    q = (g.quat_wxyz + rng.normal(0.0, 0.05, (n, 4))).astype(np.float32)
    dens = (g.density * np.exp(rng.normal(0.0, 0.1, n))).astype(np.float32)
    em = np.clip(w.emission + rng.normal(0.0, 0.05, (n, 3)), 0.0, 1.0).astype(np.float32)
    return Gaussians(mean, ls, q, dens, None, scale_is_log=True), em


def serving_scenes(sizes=(50_000, 100_000, 250_000, 500_000), seeds=(1, 2, 3, 4), env_size=(2048, 1024)) -> tuple:
    """([Gaussians per scene], sigma_multiplier, environment image) of the serving workload."""
    return [showcase_gaussians(n, s) for n, s in zip(sizes, seeds)], 7.5, procedural_env(*env_size)
