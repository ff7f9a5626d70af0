"""Builds libvolprim_b200.so (the C-ABI library of include/volprim_b200.h) in-tree for sm_100a.

Each csrc/*.cu is compiled by nvcc to an object (in parallel, skipped when up to date) and the
objects are linked into volprim_b200/_lib/libvolprim_b200.so.  Run as a script or call build().
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OBJ = HERE / "build"
LIBDIR = HERE / "volprim_b200" / "_lib"
LIB = LIBDIR / "libvolprim_b200.so"
APP = HERE / "app" / "vp_render.cpp"
APP_BIN = LIBDIR / "vp_render"
INCLUDE = HERE.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
    "-Xptxas", "-warn-spills",
]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libvolprim_b200.so")


def _deps() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [INCLUDE / "volprim_b200.h"]


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def _compile(nvcc: str, src: Path, extra: list[str]) -> tuple[Path, str]:
    obj = OBJ / (src.stem + ".o")
    cmd = [nvcc, *ARCH, *NVCC_FLAGS, *extra, "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, verbose: bool = False, extra_flags: list[str] | None = None) -> Path:
    """extra_flags (or the space-separated VP_NVCC_FLAGS environment variable) are appended to
    every nvcc compile, e.g. -DVP_WARP_MIN_BLOCKS=3; changing them needs force=True."""
    nvcc = _nvcc()
    if extra_flags is None:
        extra_flags = os.environ.get("VP_NVCC_FLAGS", "").split()
    OBJ.mkdir(parents=True, exist_ok=True)
    LIBDIR.mkdir(parents=True, exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    deps = _deps()
    todo = [s for s in sources if force or _stale(OBJ / (s.stem + ".o"), [s, *deps])]
    if todo:
        with cf.ThreadPoolExecutor(max_workers=min(len(todo), os.cpu_count() or 4)) as ex:
            for obj, log in ex.map(lambda s: _compile(nvcc, s, extra_flags or []), todo):
                if verbose and log.strip():
                    print(log, file=sys.stderr)
    objs = [OBJ / (s.stem + ".o") for s in sources]
    if force or todo or _stale(LIB, objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    build_app(force=force)
    return LIB


def build_app(force: bool = False) -> Path:
    """Compiles the vp_render command-line program (app/vp_render.cpp) against the C ABI only;
    it finds libvolprim_b200.so beside itself through an $ORIGIN run path."""
    if force or _stale(APP_BIN, [APP, APP.parent / "mitsuba_scene.h", INCLUDE / "volprim_b200.h", LIB]):
        cxx = shutil.which("g++") or shutil.which("c++")
        if cxx is None:
            raise RuntimeError("a C++ compiler (g++) is required to build vp_render")
        cmd = [cxx, "-std=c++17", "-O2", "-Wall", "-I", str(INCLUDE), str(APP), "-L", str(LIBDIR),
               "-lvolprim_b200", "-Wl,-rpath,$ORIGIN", "-o", str(APP_BIN)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"vp_render build failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return APP_BIN


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
