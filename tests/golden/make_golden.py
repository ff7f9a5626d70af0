"""Generates tests/golden/reference_pin.json from the reference's OWN code.

The reference's host-compilable headers (Primitive constructor and whitening transforms,
include/thesis/device/params/primitive.h:70-122; point_inside_bvh_bound,
include/thesis/common/geometry/intersection.h:56-61; host camera build,
include/thesis/host/params/camera.h:32-150; morton3D, include/thesis/host/utils/math.h:103-131;
the adaptive-sampling constants, device/core/constants.cuh:196-211) and its test runner's scenes
(test/scenes/geometric_validation.cpp) are compiled by oracle/Makefile into oracle/_ref/libref_pin.so; this script calls them on fixed
inputs and stores inputs and outputs (float32 bit patterns, so comparisons are exact).  It also
stores the single-Gaussian closed form of experiments/mitsuba-reference/single_gaussian_analytic.py
:78-80 (with the renderer's 3-sigma truncation) and the published PCG32 test vector.

Run from the repository root (needs the reference sources, so only where they are mounted):
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import math
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path[:0] = [str(ROOT / "oracle"), str(ROOT / "cuda-volprim_b200")]

import oracle as O  # noqa: E402
from volprim_b200 import scenes  # noqa: E402


def bits(a) -> list[int]:
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).reshape(-1).tolist()


def f32p(a):
    return O._p(O._f(a))


def primitive_cases():
    rng = np.random.default_rng(2024)
    g = scenes.absorption_gaussians(256, 0)
    cases = []
    for i in range(24):  # the 256-Gaussian absorption workload's first Gaussians
        cases.append((g.mean[i], g.scale[i], g.quat_wxyz[i], rng.uniform(0, 1, 3), float(g.density[i])))
    half = 0.5 * math.radians(30.0)  # SG_TRANSFORMED (test/scenes/single_gaussian.cpp:128-139)
    cases.append(((0, 0, 0), (1.0, 0.5, 0.75), (math.cos(half), 0, 0, math.sin(half)), (0.9, 0.9, 0.9), 7.5))
    cases.append(((0, 0, 0), (1, 1, 1), (1, 0, 0, 0), (0, 0, 0), 7.5))
    cases.append(((0.3, -0.2, 1.7), (0.02, 0.3, 0.004), (2.0, -1.0, 0.5, 3.0), (1, 0.5, 0.25), 0.125))
    cases.append(((-5.0, 4.0, 2.5), (3.0, 2.0, 1.0), (0.1, 0.2, 0.3, 0.4), (0.2, 0.4, 0.6), 1e3))
    for _ in range(8):
        q = rng.normal(size=4)
        cases.append((rng.uniform(-2, 2, 3), np.exp(rng.normal(math.log(0.05), 0.8, 3)), q * rng.uniform(0.5, 2.0),
                      rng.uniform(0, 1, 3), float(np.exp(rng.normal(0, 1)))))
    return cases


def radiance_samples(rng, n):
    """Path-tracer-like per-sample radiance: mostly log-normal, some zero paths, rare fireflies."""
    L = np.exp(rng.normal(-1.0, 1.0, (n, 3))) * (rng.uniform(size=(n, 1)) < 0.8)
    L[rng.uniform(size=n) < 0.02] *= 300.0
    return L.astype(np.float32)


def adaptive_cases(R):
    """Adaptive-sampling constants (device/core/constants.cuh:196-211), Welford sequences
    (raygen.cuh:214-222) and convergence statistics (raygen.cuh:56-63) from the reference's
    own operators."""
    k4 = np.empty(4, np.float32)
    R.ref_adaptive_constants(O._p(k4))
    rng = np.random.default_rng(99)
    io = np.empty(6, np.float32)
    welford, states = [], []
    for n in (1, 2, 5, 33, 100, 300):
        L = radiance_samples(rng, n)
        io[:] = 0.0
        for k in range(n):
            R.ref_welford_step(f32p(L[k]), k + 1, O._p(io))
        welford.append({"L": bits(L), "out": bits(io)})
        if n >= 2:
            states.append((io[:3].copy(), io[3:].copy(), n))
    for n in (2, 3, 16, 32, 64, 1000, (1 << 24) + 3):  # synthetic states
        mean = np.exp(rng.normal(-1.0, 1.0, 3)).astype(np.float32)
        m2 = (mean * mean * rng.uniform(0.0, 0.2, 3) * (n - 1)).astype(np.float32)
        states.append((mean, m2, n))
    tiny = np.float32(1e-7)
    states += [  # edges: a black channel (mean below 1e-6), constant samples (M2 = 0), and a
        # rounding-negative M2 (a NaN error) in the first and in the last channel
        (np.array([0.5, 0.0, 2e-7], np.float32), np.array([0.01, 0.0, 1e-12], np.float32), 40),
        (np.array([0.3, 0.3, 0.3], np.float32), np.zeros(3, np.float32), 50),
        (np.array([0.3, 0.2, 0.1], np.float32), np.array([-tiny, 0.02, 0.01], np.float32), 40),
        (np.array([0.3, 0.2, 0.1], np.float32), np.array([0.02, 0.01, -tiny], np.float32), 40),
    ]
    e4 = np.empty(4, np.float32)
    errors = []
    for mean, m2, n in states:
        R.ref_adaptive_error(f32p(mean), f32p(m2), n, O._p(e4))
        errors.append({"mean": bits(mean), "m2": bits(m2), "count": int(n), "err": bits(e4)})
    return {"enable": bool(k4[0]), "min_samples": int(k4[1]), "threshold": bits([k4[2]])[0],
            "min_luminance": bits([k4[3]])[0], "welford": welford, "errors": errors}


def scene_rows_digest(rows: np.ndarray) -> str:
    """sha256 of a scene's (count, 14) float32 rows: centre, forward rotation (w, x, y, z),
    scale, albedo, optical thickness."""
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(rows, np.float32).tobytes()).hexdigest()


def validation_scene_digests(R):
    """The test runner's geometric validation and stress scenes (test/scenes/
    geometric_validation.cpp, compiled into the pin library): name, Gaussian count and the digest
    of each scene's rows."""
    import ctypes as C
    R.ref_validation_scene.argtypes = [C.c_int, C.c_char_p, C.c_int, C.POINTER(C.c_float), C.c_int]
    name = C.create_string_buffer(64)
    scenes = []
    for i in range(R.ref_validation_scene_count()):
        n = R.ref_validation_scene(i, name, 64, None, 0)
        rows = np.zeros((max(n, 1), 14), np.float32)
        R.ref_validation_scene(i, name, 64, rows.ctypes.data_as(C.POINTER(C.c_float)), n)
        scenes.append({"name": name.value.decode(), "count": int(n), "sha256": scene_rows_digest(rows[:n])})
    return scenes


def main():
    O.build()
    R = O.ref_lib()
    if R is None:
        raise SystemExit("oracle/_ref/libref_pin.so is missing: the reference sources are needed")
    out = {"source": "reference headers compiled by oracle/Makefile (oracle/ref_pin.cpp)"}
    prims = []
    rec = np.empty(20, np.float32)
    tr = np.empty(7, np.float32)
    rng = np.random.default_rng(7)
    for (m, s, q, a, M) in primitive_cases():
        R.ref_primitive(f32p(m), f32p(s), f32p(q), f32p(a), float(np.float32(M)), O._p(rec))
        pts = []
        for _ in range(4):
            pos = np.asarray(m, np.float32) + rng.normal(0, 2.0 * float(np.max(s)), 3).astype(np.float32)
            d = rng.normal(size=3)
            d = (d / np.linalg.norm(d)).astype(np.float32)
            R.ref_transform(f32p(m), f32p(s), f32p(q), float(np.float32(M)), f32p(pos), f32p(d), O._p(tr))
            pts.append({"pos": bits(pos), "dir": bits(d), "out": bits(tr)})
        prims.append({"mean": bits(m), "scale": bits(s), "quat_wxyz": bits(q), "albedo": bits(a),
                      "density": bits([M])[0], "record": bits(rec), "transforms": pts})
    out["primitives"] = prims
    cams = []
    cam_cases = [
        ("absorption_256 negz", (0, 0, -3.5), (0, 0, 0), (0, 1, 0), 40.0, 2.0, 0, 128, 128),
        ("default", (0, 0, -1), (0, 0, 0), (0, 1, 0), 90.0, 2.0, 0, 1000, 750),
        ("asset diag", (2.1, 1.75, -2.1), (0, 0, 0), (0, 1, 0), 40.0, 2.0, 0, 512, 512),
        ("asset posy", (0, 3.5, 0), (0, 0, 0), (0, 0, 1), 40.0, 2.0, 0, 512, 512),
        ("showcase 900x600", (0.7, 0.3, -3.2), (0.1, -0.1, 0.2), (0, 1, 0), 35.0, 2.0, 0, 900, 600),
        ("single_gaussian ortho", (0, 0, -5), (0, 0, 0), (0, 1, 0), 90.0, 6.0, 1, 256, 256),
        ("cluster n5 ortho", (0, 0, -6), (0, 0, 0), (0, 1, 0), 90.0, 8.0, 1, 256, 256),
        ("ortho oblique", (3, 2, -4), (0, 0.5, 0), (0, 1, 0), 90.0, 4.5, 1, 320, 200),
    ]
    c16 = np.empty(16, np.float32)
    for name, eye, at, up, fov, oh, ortho, W, H in cam_cases:
        R.ref_camera(f32p(eye), f32p(at), f32p(up), float(fov), float(oh), int(ortho), W, H, O._p(c16))
        cams.append({"name": name, "eye": bits(eye), "lookat": bits(at), "up": bits(up), "vfov": bits([fov])[0],
                     "ortho_height": bits([oh])[0], "orthographic": ortho, "width": W, "height": H,
                     "out": bits(c16)})
    out["cameras"] = cams
    mort = []
    smin = np.array([-1.0, -0.5, -0.7], np.float32)
    inv = (1.0 / np.array([2.0, 1.0, 1.4], np.float32)).astype(np.float32)
    for p in rng.uniform([-1.1, -0.6, -0.8], [1.1, 0.6, 0.8], (32, 3)).astype(np.float32):
        mort.append({"pos": bits(p), "code": int(R.ref_morton3d(f32p(p), f32p(smin), f32p(inv)))})
    out["morton"] = {"scene_min": bits(smin), "inv_extent": bits(inv), "cases": mort}
    # closed form: unit isotropic Gaussian of mass M, 3-sigma truncated chord at distance d
    M = 7.5
    ds = np.linspace(0.0, 2.99, 24)
    out["single_gaussian"] = {"mass": M, "d": ds.tolist(),
                              "tau": [M / (2 * math.pi) * math.exp(-d * d / 2) * math.erf(math.sqrt((9 - d * d) / 2))
                                      for d in ds]}
    # PCG32 reference implementation demo (pcg32_srandom_r(42, 54)): first six outputs
    out["pcg32"] = {"seed": 42, "sequence": 54,
                    "outputs": [0xa15c02b7, 0x7b47f409, 0xba1d3330, 0x83d2f293, 0xbfa4784b, 0xcbed606e]}
    out["adaptive"] = adaptive_cases(R)
    out["validation_scenes"] = validation_scene_digests(R)
    path = Path(__file__).resolve().parent / "reference_pin.json"
    path.write_text(json.dumps(out, indent=1))
    print(f"wrote {path} ({path.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
