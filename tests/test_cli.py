"""The vp_render command-line program (cuda-volprim_b200/app/vp_render.cpp): the reference
renderer's options (src/thesis/host/app/config.cpp:15-50) and its default scene and camera
(src/thesis/host/main.cpp:21-30, camera.h getDefaultCamera) over the C ABI, writing the image as a
vertically flipped EXR as Image::save does.

CPU: option parsing and its errors (they are reported before any CUDA call).
GPU: the EXR the program writes equals the image the library renders through the Python API for
the same scene, environment, camera and parameters (the same render call with the same seeds, so
the comparison is exact up to the order-independent FP32 sums: 1e-6 relative + 1e-7).
"""
import subprocess

import numpy as np
import pytest

import build_lib
import volprim_b200 as vp
from volprim_b200 import io as vio
from volprim_b200 import scenes
from test_io import read_exr, rgbe_encode, write_hdr


@pytest.fixture(scope="module")
def exe():
    if not build_lib.LIB.exists():
        pytest.skip("libvolprim_b200.so is not built")
    return str(build_lib.build_app())


def run(exe, *args, cwd=None):
    return subprocess.run([exe, *map(str, args)], capture_output=True, text=True, cwd=cwd, timeout=600)


@pytest.mark.parametrize("args, message", [
    (["--bogus"], "unknown option --bogus"),
    (["--width"], "needs 1 value"),
    (["--eye", "0", "1"], "needs 3 value"),
    (["--width", "12x"], "not an unsigned integer"),
    (["--phase-g", "0.9995"], "--phase-g must be in"),
    (["--rr-max-survival", "1.5"], "--rr-max-survival must be in"),
    (["--firefly-clamp", "-1"], "--firefly-clamp must be non-negative"),
    (["--max-depth", "0"], "--max-depth must be positive"),
    (["--adaptive-threshold", "-0.1"], "--adaptive-threshold must be non-negative"),
    (["--adaptive-min-samples", "x"], "not an unsigned integer"),
    (["--engine", "optix"], "unknown engine optix"),
    (["--precision", "half"], "unknown precision half"),
])
def test_cli_option_errors(exe, args, message):
    r = run(exe, *args)
    assert r.returncode == 1
    assert message in r.stderr


def test_cli_help(exe):
    r = run(exe, "--help")
    assert r.returncode == 0


def flipped_exr(path):
    names, _, img = read_exr(path)
    assert names == ["B", "G", "R"]
    return img[::-1, :, ::-1]  # rows back to the render's order, channels to R, G, B


def near(a, b):
    return np.abs(a - b) <= 1e-6 * np.abs(b) + 1e-7


@pytest.mark.gpu
def test_cli_default_scene(exe, vp_ctx, tmp_path):
    out = tmp_path / "default.exr"
    r = run(exe, "--output", out, "--width", 48, "--height", 36, "--samples_per_pixel", 8, "--seed", 5,
            "--module_blob", "ignored.optixir", "--raygen", "__raygen__rg")
    assert r.returncode == 0, r.stderr
    assert "rendered 48x36 x 8 spp of 1 Gaussians" in r.stdout
    g = vp.Gaussians(mean=np.zeros((1, 3), np.float32), scale=np.full((1, 3), 0.5, np.float32),
                     quat_wxyz=np.array([[1, 0, 0, 0]], np.float32), density=np.array([0.5], np.float32),
                     albedo=np.array([[0.5, 0.0, 0.5]], np.float32))
    cfg = vp.Config(num_samples_per_pixel=8, image_width=48, image_height=36, seed=5)
    want = vp.Renderer(cfg, vp.Scene(vp_ctx, g), ctx=vp_ctx).render()
    got = flipped_exr(out)
    assert got.shape == (36, 48, 3)
    assert np.all(near(got, want[..., :3]))
    assert want[..., :3].max() > 0.05  # the purple Gaussian is in view


@pytest.mark.gpu
def test_cli_ply_env_and_options(exe, vp_ctx, tmp_path):
    g = scenes.showcase_gaussians(3000, 11)
    ply = tmp_path / "scene.ply"
    vio.save_ply(ply, vp.Gaussians(g.mean, np.log(g.scale).astype(np.float32), g.quat_wxyz, g.density, g.albedo,
                                   scale_is_log=True))
    env_rgb = scenes.procedural_env(64, 32, sun_radiance=50.0, sun_radius_deg=8.0)
    hdr = tmp_path / "env.hdr"
    write_hdr(hdr, rgbe_encode(env_rgb))
    out = tmp_path / "scene.exr"
    eye, look, up = (2.2, 1.0, -2.5), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0)
    r = run(exe, "--output", out, "--width", 40, "--height", 30, "--samples_per_pixel", 6, "--seed", 9,
            "--ply", ply, "--env_map", hdr, "--sigma-multiplier", 4.0, "--albedo", 0.2, 0.5, 0.8,
            "--phase-g", 0.3, "--max-depth", 12, "--rr-depth", 3, "--rr-max-survival", 0.9,
            "--filter-width", 0.6, "--ris", "--ris-candidates", 4, "--measure-caps",
            "--eye", *eye, "--lookat", *look, "--up", *up, "--vfov", 50)
    assert r.returncode == 0, r.stderr
    assert "max hits per ray" in r.stdout
    cfg = vp.Config(num_samples_per_pixel=6, image_width=40, image_height=30, seed=9, hg_g=0.3, max_bounces=12,
                    rr_depth=3, rr_max_survival=0.9, pixel_filter_stddev=0.6, use_ris=True, ris_num_candidates=4,
                    measure_caps=True)
    scene = vp.Scene(vp_ctx, vio.load_ply(ply, albedo_override=(0.2, 0.5, 0.8)), 4.0)
    env = vp.Environment(vp_ctx, rgb=vio.load_hdr(hdr))
    cam = vp.Camera.perspective(eye, look, up, 50.0)
    want = vp.Renderer(cfg, scene, camera=cam, env=env, ctx=vp_ctx).render()
    got = flipped_exr(out)
    assert np.all(near(got, want[..., :3]))
    assert want[..., :3].mean() > 1e-3


@pytest.mark.gpu
def test_cli_orthographic_and_engines(exe, vp_ctx, tmp_path):
    imgs = {}
    for engine in ("wavefront", "warp"):
        out = tmp_path / f"{engine}.exr"
        r = run(exe, "--output", out, "--width", 32, "--height", 32, "--samples_per_pixel", 4,
                "--ortho-height", 1.5, "--engine", engine, "--precision", "fast")
        assert r.returncode == 0, r.stderr
        imgs[engine] = flipped_exr(out)
    # the two BVH32 engines run the same per-path code and seeds
    assert np.allclose(imgs["wavefront"], imgs["warp"], rtol=1e-5, atol=1e-6)
    g = vp.Gaussians(mean=np.zeros((1, 3), np.float32), scale=np.full((1, 3), 0.5, np.float32),
                     quat_wxyz=np.array([[1, 0, 0, 0]], np.float32), density=np.array([0.5], np.float32),
                     albedo=np.array([[0.5, 0.0, 0.5]], np.float32))
    cfg = vp.Config(num_samples_per_pixel=4, image_width=32, image_height=32, precision="fast")
    cam = vp.Camera.orthographic_camera((0, 0, -1), (0, 0, 0), (0, 1, 0), 1.5)
    want = vp.Renderer(cfg, vp.Scene(vp_ctx, g), camera=cam, ctx=vp_ctx).render()
    assert np.all(near(imgs["wavefront"], want[..., :3]))


# A Mitsuba scene description in the form the reference's parser reads
# (src/thesis/host/utils/mitsuba_parser.cpp:39-149): camera blocks of a Python dict with an
# optional resolution and a T().look_at(...) call that may span lines.
MITSUBA_INIT = """\
OBJECTS = {'cloud': {'type': 'ply', 'extent': 2.5}}
SENSORS = {
    'cam_0000': {
        'type': 'orthographic',
        'width': 40,
        'height': 30,
        'to_world': T().look_at(origin=[0.0, 0.0, -4.0], target=[0.0, 0.0, 0.0],
                                up=[0.0, 1.0, 0.0]),
    },
    'cam_0001': {
        'type': 'orthographic',
        'to_world': T().look_at(
            origin=[3.5, 1.25e+0, -2.0],
            target=[0.1, -0.2, 0.3],
            up=[0.0, 1.0, 0.0]),
    },
    'cam_0002': {
        'to_world': T().look_at(origin=[1.0, 2.0, 3.0], target=[0.0, 0.0, 0.0]),
    },
    'cam_0003': {
        'height': 16,
        'to_world': T().look_at(origin=[-2.0, 0.5, 2.0], target=[0.0, 0.0, 0.0], up=[0, 1, 0]),
    },
}
"""


def mitsuba_files(tmp_path, init=MITSUBA_INIT, args='{"cam_res": 24, "spp": 64}'):
    py, js = tmp_path / "__init__.py", tmp_path / "args.json"
    py.write_text(init)
    js.write_text(args)
    return py, js


def listed(stdout):
    rows = []
    for ln in stdout.splitlines():
        t = ln.split()
        f32 = lambda v: tuple(np.float32(x) for x in v)  # %.9g round-trips a float32
        rows.append({"index": int(t[0]), "name": t[1], "res": tuple(map(int, t[2].split("x"))),
                     "origin": f32(t[4:7]), "target": f32(t[8:11]), "up": f32(t[12:15]),
                     "ortho_height": np.float32(t[16])})
    return rows


def test_cli_mitsuba_cameras_parsed(exe, tmp_path):
    """Camera blocks, per-camera resolutions over the args.json default, look-at blocks over
    several lines, a block without `up` dropped (as the reference drops it), and the orthographic
    viewport height 2 / aspect of createOrthographicCamera (mitsuba_parser.cpp:213-225)."""
    py, js = mitsuba_files(tmp_path)
    r = run(exe, "--mitsuba-scene", py, js, "--list-cameras")
    assert r.returncode == 0, r.stderr
    rows = listed(r.stdout)
    assert [c["name"] for c in rows] == ["cam_0000", "cam_0001", "cam_0003"]
    assert [c["res"] for c in rows] == [(40, 30), (24, 24), (24, 16)]
    assert rows[0]["origin"] == (0.0, 0.0, -4.0) and rows[0]["up"] == (0.0, 1.0, 0.0)
    assert rows[1]["origin"] == (3.5, 1.25, -2.0)
    assert rows[1]["target"] == tuple(np.float32(x) for x in ("0.1", "-0.2", "0.3"))
    for c in rows:
        w, h = c["res"]
        assert c["ortho_height"] == np.float32(2.0) / (np.float32(w) / np.float32(h))
    r = run(exe, "--mitsuba-scene", py, js, "--list-cameras", "--camera", 1)
    assert r.returncode == 0 and [c["name"] for c in listed(r.stdout)] == ["cam_0001"]
    _, js2 = mitsuba_files(tmp_path, args="{}")  # no cam_res: 800 x 800
    r = run(exe, "--mitsuba-scene", py, js2, "--list-cameras")
    assert [c["res"] for c in listed(r.stdout)] == [(40, 30), (800, 800), (800, 16)]


@pytest.mark.parametrize("case, message", [
    ("no_args_json", "failed to open args.json"),
    ("no_cameras", "no cameras found"),
    ("camera_out_of_range", "--camera 9 out of range (3 cameras)"),
    ("list_without_scene", "--list-cameras and --camera need --mitsuba-scene"),
])
def test_cli_mitsuba_errors(exe, tmp_path, case, message):
    py, js = mitsuba_files(tmp_path, init="SENSORS = {}\n" if case == "no_cameras" else MITSUBA_INIT)
    args = {"no_args_json": ["--mitsuba-scene", py, tmp_path / "missing.json", "--list-cameras"],
            "no_cameras": ["--mitsuba-scene", py, js, "--list-cameras"],
            "camera_out_of_range": ["--mitsuba-scene", py, js, "--list-cameras", "--camera", 9],
            "list_without_scene": ["--list-cameras"]}[case]
    r = run(exe, *args)
    assert r.returncode == 1
    assert message in r.stderr


@pytest.mark.gpu
def test_cli_mitsuba_multiview(exe, vp_ctx, tmp_path):
    """The harness renders each camera at its resolution to OUTPUT_DIR/NNNN.exr; each image is the
    API's render through the same orthographic camera."""
    py, js = mitsuba_files(tmp_path)
    out = tmp_path / "views"
    r = run(exe, "--mitsuba-scene", py, js, "--output-dir", out, "--samples_per_pixel", 4, "--seed", 3)
    assert r.returncode == 0, r.stderr
    g = vp.Gaussians(mean=np.zeros((1, 3), np.float32), scale=np.full((1, 3), 0.5, np.float32),
                     quat_wxyz=np.array([[1, 0, 0, 0]], np.float32), density=np.array([0.5], np.float32),
                     albedo=np.array([[0.5, 0.0, 0.5]], np.float32))
    scene = vp.Scene(vp_ctx, g)
    for i, c in enumerate(listed(run(exe, "--mitsuba-scene", py, js, "--list-cameras").stdout)):
        w, h = c["res"]
        cam = vp.Camera.orthographic_camera(c["origin"], c["target"], c["up"], c["ortho_height"])
        cfg = vp.Config(num_samples_per_pixel=4, image_width=w, image_height=h, seed=3)
        want = vp.Renderer(cfg, scene, camera=cam, ctx=vp_ctx).render()[..., :3]
        got = flipped_exr(out / f"{i:04d}.exr")
        assert got.shape == (h, w, 3)
        assert np.all(near(got, want)), i
        assert want.max() > 0.05
    assert sorted(p.name for p in out.iterdir()) == ["0000.exr", "0001.exr", "0002.exr"]
