"""The reference's geometric validation scenes as regression fixtures.

The scenes of the reference's test runner (test/scenes/geometric_validation.cpp; listed by
get_validation_test_scenes and get_stress_test_scenes): a few hand-placed Gaussians each, chosen
to hit one edge of the method -- coincident and nested Gaussians, a camera inside or at the edge
of one, 64 and 65 Gaussians on one ray (the reference's 128-entry hit buffer), extreme scales and
optical thicknesses, rotations with w = 0, an empty scene.  The runner renders them through
app::Renderer with the default camera (eye (0, 0, -1) looking at the origin, vertical field of
view 90 degrees, camera.h getDefaultCamera) and builds each Gaussian with
Primitive::from_forward_quat(centre, rotation, scale, albedo, optical_thickness), the optical
thickness given as a peak extinction times (2 pi)^(3/2) * sx * sy * sz (sigma_dsyg,
geometric_validation.cpp:16-19).  The runner applies no sigma multiplier to them.

Each scene here is a Gaussians record with density = that optical thickness (the library's mass
convention, the same quantity), built from a table of (centre, scale, albedo, peak extinction,
rotation) rows.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from volprim_b200.api import Camera, Gaussians

_ROOT_TWO_PI = np.float32(2.5066282746)  # math::ROOT_TWO_PI_F
_TWO_PI = np.float32(2.0) * np.float32(np.pi)  # math::TWO_PI_F (float32 product)
IDENTITY = (1.0, 0.0, 0.0, 0.0)  # (w, x, y, z)

RED, GREEN, BLUE = (1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0)
YELLOW, CYAN, MAGENTA = (1.0, 1.0, 0.0), (0.0, 1.0, 1.0), (1.0, 0.0, 1.0)


def optical_thickness(peak: float, scale) -> np.float32:
    """Peak extinction -> the mass-normalised optical thickness, in the reference's float32
    order: peak * sqrt(2 pi) * 2 pi * (sx * sy * sz)."""
    s = np.asarray(scale, np.float32)
    return np.float32(np.float32(np.float32(peak) * _ROOT_TWO_PI) * _TWO_PI) * np.float32(
        np.float32(s[0] * s[1]) * s[2])


@dataclass
class ValidationScene:
    name: str
    description: str
    gaussians: Gaussians


def _scene(name: str, description: str, rows) -> ValidationScene:
    """rows: (centre, scale, albedo, peak extinction[, rotation (w, x, y, z)])."""
    n = len(rows)
    mean = np.zeros((n, 3), np.float32)
    scale = np.zeros((n, 3), np.float32)
    alb = np.zeros((n, 3), np.float32)
    quat = np.zeros((n, 4), np.float32)
    dens = np.zeros(n, np.float32)
    for i, row in enumerate(rows):
        c, s, a, peak = row[:4]
        mean[i], scale[i], alb[i] = c, s, a
        quat[i] = row[4] if len(row) > 4 else IDENTITY
        dens[i] = optical_thickness(peak, s)
    return ValidationScene(name, description, Gaussians(mean, scale, quat, dens, alb))


def _iso(s: float):
    return (s, s, s)


F = np.float32  # positions and colours below are computed in float32, as the reference does


def _grid(name, description, nx, ny, spacing, s, z=5.0, peak=10.0):
    """create_grid_stress_test: an nx x ny grid centred on the z axis at depth z, albedo
    (x / (nx - 1), 0.5, y / (ny - 1))."""
    sp = F(spacing)
    ox, oy = -(F(nx - 1) * sp) * F(0.5), -(F(ny - 1) * sp) * F(0.5)
    rows = [((ox + F(x) * sp, oy + F(y) * sp, z), _iso(s), (F(x) / F(nx - 1), 0.5, F(y) / F(ny - 1)), peak)
            for y in range(ny) for x in range(nx)]
    return _scene(name, description, rows)


def _hue(i: int):
    h = F(i) / F(100.0)
    if h < F(0.5):
        return (1.0, h * F(2.0), 0.0)
    return (F(1.0) - (h - F(0.5)) * F(2.0), 1.0, (h - F(0.5)) * F(2.0))


def validation_scenes() -> list[ValidationScene]:
    """The 36 scenes of get_validation_test_scenes, in its order."""
    q8 = (0.92388, 0.0, 0.0, 0.382683)   # pi/4 about z
    q4 = (0.707107, 0.0, 0.0, 0.707107)  # pi/2 about z
    rod = (1.0, 0.3, 0.3)
    return [
        _scene("single_purple", "one purple Gaussian (the blend coincident_surfaces should give)",
               [((0, 0, 0), _iso(0.5), (0.5, 0.0, 0.5), 0.5)]),
        _scene("coincident_surfaces", "red and blue Gaussians at the same place",
               [((0, 0, 0), _iso(0.5), RED, 0.5), ((0, 0, 0), _iso(0.5), BLUE, 0.5)]),
        _scene("partial_overlap", "two Gaussians overlapping in part",
               [((-0.3, 0, 0), _iso(0.5), BLUE, 0.5), ((0.3, 0, 0), _iso(0.5), RED, 0.5)]),
        _scene("total_overlap", "a small dense Gaussian inside a large thin one",
               [((0, 0, 0), _iso(1.0), RED, 0.3), ((0, 0, 0), _iso(0.3), BLUE, 0.8)]),
        _scene("depth_ordering", "three Gaussians one behind the other",
               [((0, 0, 1), _iso(0.4), RED, 1.5), ((0, 0, 3), _iso(0.4), GREEN, 1.5),
                ((0, 0, 5), _iso(0.4), BLUE, 1.5)]),
        _scene("camera_inside", "the camera inside one large Gaussian",
               [((0, 0, 0), _iso(5.0), RED, 0.2)]),
        _scene("non_overlapping", "three separate Gaussians",
               [((-1.5, 0, 0), _iso(0.4), RED, 0.5), ((0, 0, 0), _iso(0.4), GREEN, 0.5),
                ((1.5, 0, 0), _iso(0.4), BLUE, 0.5)]),
        _scene("transform_scale", "four scales, one stretched along x",
               [((-1.0, 0.5, 3.0), _iso(0.2), RED, 0.5), ((0.0, 0.5, 0.0), _iso(0.5), GREEN, 0.5),
                ((1.0, 0.5, 0.0), _iso(1.0), BLUE, 0.5), ((0.0, -0.8, 0.0), rod, YELLOW, 0.5)]),
        _scene("transform_rotation", "one ellipsoid at rotations 0, pi/4 and pi/2 about z",
               [((-1.5, 0, 0), rod, RED, 0.5), ((0, 0, 0), rod, GREEN, 0.5, q8),
                ((1.5, 0, 0), rod, BLUE, 0.5, q4)]),
        _scene("transform_translation", "one Gaussian on a 3 x 3 grid of positions",
               [((x, y, 0), _iso(0.4), CYAN, 0.5) for y in (-1, 0, 1) for x in (-1, 0, 1)]),
        _scene("many_gaussians", "a 10 x 10 grid of small Gaussians at depth 5",
               [(((x - 4.5) * 0.25, (y - 4.5) * 0.25, 5.0), _iso(0.1), _hue(y * 10 + x), 2.0)
                for y in range(10) for x in range(10)]),
        _scene("nested_structure", "three concentric Gaussians",
               [((0, 0, 0), _iso(1.5), RED, 0.25), ((0, 0, 0), _iso(1.0), GREEN, 0.3),
                ((0, 0, 0), _iso(0.5), BLUE, 0.6)]),
        _scene("tangent_rays", "a Gaussian whose 3-sigma box holds the camera at its side",
               [((1, 0, 0), _iso(0.8), YELLOW, 0.5)]),
        _scene("empty_scene", "no Gaussians: only the environment", []),
        _scene("hit_buffer_at_capacity", "64 thin Gaussians on the optical axis (128 crossings)",
               [((0, 0, i * 0.5 + 1.0), _iso(0.3), RED, 0.05) for i in range(64)]),
        _scene("hit_buffer_overflow", "65 thin Gaussians on the optical axis (130 crossings)",
               [((0, 0, i * 0.5 + 1.0), _iso(0.3), GREEN, 0.05) for i in range(65)]),
        _scene("ray_at_exact_boundary", "the camera one sigma from a unit Gaussian's centre",
               [((0, 0, 0), _iso(1.0), YELLOW, 0.3)]),
        _scene("all_behind_camera", "five Gaussians behind the camera",
               [((i - 2, 0.0, -5.0 - i), _iso(0.5), MAGENTA, 0.5) for i in range(5)]),
        _scene("extreme_anisotropic_scale", "needles and a pancake with 100:1 axes",
               [((-1.0, 0.5, 3.0), (5.0, 0.05, 0.05), RED, 0.3), ((1.0, 0.5, 3.0), (1.0, 0.01, 1.0), BLUE, 0.3),
                ((0.0, -0.5, 3.0), (0.05, 0.05, 5.0), GREEN, 0.3)]),
        _scene("extreme_small_scale", "a 3 x 3 grid of Gaussians of scale 0.01",
               [((x * 0.1, y * 0.1, 2.0), _iso(0.01), YELLOW, 1.0) for y in (-1, 0, 1) for x in (-1, 0, 1)]),
        _scene("extreme_large_scale", "a Gaussian of scale 100 around a small one",
               [((0, 0, 50), _iso(100.0), CYAN, 0.01), ((0, 0, 3), _iso(0.5), RED, 0.5)]),
        _scene("near_coincident_surfaces", "two Gaussians 1e-5 apart",
               [((0, 0, 0), _iso(0.5), RED, 0.5), ((0.00001, 0, 0), _iso(0.5), BLUE, 0.5)]),
        _scene("collinear_with_gaps", "five separate Gaussians on the optical axis",
               [((0, 0, i * 1.5 + 1.0), _iso(0.4),
                 (1.0 if i in (0, 4) else 0.0, 1.0 if i in (1, 2) else 0.0, 1.0 if i in (2, 3, 4) else 0.0), 0.5)
                for i in range(5)]),
        _scene("nested_off_center", "a small dense Gaussian near the edge of a large one",
               [((0, 0, 0), _iso(1.5), RED, 0.2), ((1, 0, 0), _iso(0.3), BLUE, 0.8)]),
        _scene("chain_overlaps", "A overlaps B, B overlaps C, A and C apart",
               [((-0.8, 0, 0), _iso(0.5), BLUE, 0.5), ((0, 0, 0), _iso(0.5), GREEN, 0.5),
                ((0.8, 0, 0), _iso(0.5), RED, 0.5)]),
        _scene("rotation_180_degrees", "an ellipsoid turned by pi about z (w = 0)",
               [((-1, 0, 0), rod, BLUE, 0.5), ((1, 0, 0), rod, RED, 0.5, (0.0, 0.0, 0.0, 1.0))]),
        _scene("high_optical_thickness", "peak extinction 10: transmittance underflows",
               [((0, 0, 0), _iso(0.5), (0.8, 0.8, 0.8), 10.0)]),
        _scene("low_optical_thickness", "peak extinction 0.001: almost transparent",
               [((0, 0, 0), _iso(1.0), CYAN, 0.001)]),
        _scene("zero_albedo", "a pure absorber", [((0, 0, 0), _iso(1.0), (0.0, 0.0, 0.0), 0.5)]),
        _scene("debug_single_at_origin", "one Gaussian at the origin",
               [((0, 0, 0), _iso(0.4), CYAN, 0.5)]),
        _scene("debug_single_offset", "one Gaussian at (1, 0, 0)", [((1, 0, 0), _iso(0.4), CYAN, 0.5)]),
        _scene("debug_two_at_origin", "two Gaussians at the origin",
               [((0, 0, 0), _iso(0.4), RED, 0.5), ((0, 0, 0), _iso(0.4), BLUE, 0.5)]),
        _scene("debug_grid_2x2", "a 2 x 2 grid",
               [((x, y, 0), _iso(0.4), CYAN, 0.5) for y in (0, 1) for x in (0, 1)]),
        _scene("minimal_behind_camera", "one Gaussian behind the camera",
               [((0, 0, -2), _iso(0.5), RED, 0.5)]),
        _scene("minimal_in_front", "one Gaussian in front of the camera",
               [((0, 0, 3), _iso(0.5), GREEN, 0.5)]),
        _scene("multiple_same_z", "a 3 x 3 grid at one depth",
               [((x * 0.5, y * 0.5, 2.0), _iso(0.3), RED, 0.5) for y in (-1, 0, 1) for x in (-1, 0, 1)]),
    ]


def stress_scenes() -> list[ValidationScene]:
    """The 7 grids of get_stress_test_scenes (peak extinction 10, depth 5)."""
    return [
        _grid("stress_16_gaussians", "4 x 4 grid", 4, 4, 0.4, 0.2),
        _grid("stress_256_gaussians", "16 x 16 grid", 16, 16, 0.4, 0.2),
        _grid("stress_512_gaussians", "32 x 16 grid", 32, 16, 0.2, 0.1),
        _grid("stress_1024_gaussians", "32 x 32 grid", 32, 32, 0.2, 0.1),
        _grid("stress_2048_gaussians", "64 x 32 grid", 64, 32, 0.1, 0.05),
        _grid("stress_4096_gaussians", "64 x 64 grid", 64, 64, 0.1, 0.05),
        _grid("stress_8192_gaussians", "128 x 64 grid", 128, 64, 0.05, 0.025),
    ]


def all_scenes() -> list[ValidationScene]:
    return validation_scenes() + stress_scenes()


def runner_camera() -> Camera:
    """The camera the test runner renders these scenes with (getDefaultCamera)."""
    return Camera.default()
