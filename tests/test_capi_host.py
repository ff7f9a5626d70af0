"""CPU: the C-ABI library loads, exports every entry point include/volprim_b200.h declares, and its
host-only entry points behave (no device work is issued here)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

import volprim_b200 as vp
from volprim_b200 import _capi

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "volprim_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:vp_status|const char\*)\s+(vp_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_the_entry_points():
    names = declared_functions()
    for must in ("vp_context_create", "vp_scene_create", "vp_env_create", "vp_render", "vp_render_accumulate",
                 "vp_transmittance", "vp_albedo_at", "vp_camera_rays", "vp_normalize_accumulator",
                 "vp_last_error_string"):
        assert must in names
    assert len(names) >= 25


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(str(_capi.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    nm = subprocess.run(["nm", "-D", "--defined-only", str(_capi.LIB_PATH)], capture_output=True, text=True)
    if nm.returncode == 0:
        exported = {ln.split()[-1] for ln in nm.stdout.splitlines() if ln.strip()}
        assert set(declared_functions()) <= exported


def test_python_bindings_cover_the_header():
    assert set(declared_functions()) == set(_capi.SIGNATURES)


def test_version_and_defaults():
    mj, mn = C.c_int32(), C.c_int32()
    _capi.check(_capi.lib.vp_version(C.byref(mj), C.byref(mn)))
    assert (mj.value, mn.value) == (0, 1)
    p = _capi.vp_render_params()
    _capi.check(_capi.lib.vp_render_params_default(C.byref(p)))
    # app::Config defaults (include/thesis/host/app/config.h:30-47), BATCH_SIZE (renderer.cpp:32)
    assert (p.width, p.height, p.spp, p.seed, p.max_bounces, p.rr_depth) == (1000, 750, 1, 42, 128, 12)
    assert abs(p.rr_max_survival - 0.99) < 1e-7 and abs(p.hg_g - 0.85) < 1e-7
    assert p.firefly_clamp == 0.0 and p.pixel_filter_stddev == 0.0
    assert p.nee_mode == vp.VP_NEE_MIS and p.ris_candidates == 6 and p.batch_spp == 16
    assert p.engine == _capi.VP_ENGINE_WAVEFRONT
    # ADAPTIVE_THRESHOLD (off) and ADAPTIVE_MIN_SAMPLES (device/core/constants.cuh:202-207)
    assert p.adaptive_threshold == 0.0 and p.adaptive_min_samples == 32


def test_scene_option_defaults():
    o = _capi.vp_scene_options()
    _capi.check(_capi.lib.vp_scene_options_default(C.byref(o)))
    assert (o.wide_builder, o.binary_builder, o.leaf_max, o.wide_collapse) == (
        _capi.VP_TREE_PLOC, _capi.VP_TREE_PLOC, 24, _capi.VP_COLLAPSE_SAH)
    assert _capi.lib.vp_scene_options_default(None) == -1
    assert _capi.lib.vp_scene_create_ex(None, None, C.c_float(1.0), None, None) == -1


def test_null_arguments_are_errors_not_crashes():
    assert _capi.lib.vp_context_create(0, None) == -1
    assert b"NULL" in _capi.lib.vp_last_error_string() or _capi.lib.vp_last_error_string()
    assert _capi.lib.vp_scene_create(None, None, C.c_float(1.0), None) == -1
    assert _capi.lib.vp_render(None, None, None, None, None, 0, None) == -1
    assert _capi.lib.vp_render_params_default(None) == -1
    with pytest.raises(_capi.VpError):
        _capi.check(_capi.lib.vp_render_params_default(None))


def test_config_maps_to_c_params():
    cfg = vp.Config(num_samples_per_pixel=256, image_width=512, image_height=256, seed=9, max_bounces=64,
                    rr_depth=12, hg_g=0.0, use_ris=True, ris_num_candidates=4, engine="megakernel",
                    precision="accurate", batch_spp=8, measure_caps=True, adaptive_threshold=0.05,
                    adaptive_min_samples=16)
    p = cfg.to_c()
    assert (p.width, p.height, p.spp, p.seed, p.max_bounces) == (512, 256, 256, 9, 64)
    assert p.nee_mode == vp.VP_NEE_RIS and p.ris_candidates == 4
    assert p.engine == vp.VP_ENGINE_MEGAKERNEL and p.precision == vp.VP_PRECISION_ACCURATE
    assert p.batch_spp == 8 and p.measure == 1
    assert abs(p.adaptive_threshold - 0.05) < 1e-8 and p.adaptive_min_samples == 16


def test_struct_layouts_match_header(tmp_path):
    """Every ctypes mirror has the size and field offsets that gcc gives the header's structs."""
    structs = {"vp_gaussians": _capi.vp_gaussians, "vp_scene_info": _capi.vp_scene_info,
               "vp_camera": _capi.vp_camera, "vp_render_params": _capi.vp_render_params,
               "vp_render_stats": _capi.vp_render_stats, "vp_gaussian_grads": _capi.vp_gaussian_grads,
               "vp_server_config": _capi.vp_server_config, "vp_request": _capi.vp_request,
               "vp_server_stats": _capi.vp_server_stats, "vp_scene_options": _capi.vp_scene_options}
    lines = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void) {"]
    for name, cls in structs.items():
        lines.append(f'  printf("{name} %zu\\n", sizeof({name}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{name}.{fname} %zu\\n", offsetof({name}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    cc = subprocess.run(["gcc", "-std=c11", "-I", "/usr/local/cuda/include", str(src), "-o", str(exe)],
                        capture_output=True, text=True)
    if cc.returncode != 0:
        pytest.skip("no C compiler for the header: " + cc.stderr[:200])
    got = dict(ln.split() for ln in subprocess.run([str(exe)], capture_output=True, text=True,
                                                   check=True).stdout.splitlines())
    for name, cls in structs.items():
        assert int(got[name]) == C.sizeof(cls), name
        for fname, _ in cls._fields_:
            assert int(got[f"{name}.{fname}"]) == getattr(cls, fname).offset, f"{name}.{fname}"
    assert C.sizeof(_capi.vp_gaussians) == 56
    assert C.sizeof(_capi.vp_camera) == 48
    assert C.sizeof(_capi.vp_render_params) == 72