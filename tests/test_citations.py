"""CPU: every `file:line` citation of the reference in the boundary header, the CUDA sources, the
host package, the oracle and the design notes points at lines that exist in the reference tree.

A citation is a path ending in a source or document suffix followed by `:line` or `:a-b` (more
ranges may follow, comma-separated).  The path may be the file's path within the reference
project or any suffix of it (`primitive.h:249-318`); it must match at least one file of the
tree, and some match must be at least as long as the highest line cited.  Skipped where the
reference tree is not present (it is read only here, never at run time).
"""
import os
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
REF = Path(os.environ.get("VP_REFERENCE_TREE", str(ROOT.parent / "reference")))

SUFFIXES = r"(?:h|hpp|cuh|cu|cpp|c|py|tex|md|cmake|txt|cff|json|sh)"
CITE = re.compile(r"([A-Za-z0-9_./-]+\." + SUFFIXES + r"):(\d+(?:-\d+)?(?:\s*,\s*:?\d+(?:-\d+)?)*)")

# Files of this repository whose citations name the reference.
SOURCES = [
    *sorted((ROOT / "include").glob("*.h")),
    *sorted((ROOT / "cuda-volprim_b200" / "csrc").glob("*")),
    *sorted((ROOT / "cuda-volprim_b200" / "app").glob("*")),
    *sorted((ROOT / "cuda-volprim_b200" / "volprim_b200").glob("*.py")),
    *sorted((ROOT / "oracle").glob("*.cpp")),
    *sorted((ROOT / "oracle").glob("*.py")),
    ROOT / "DESIGN.md",
    ROOT / "INTEGRATION.md",
    ROOT / "BASELINE.md",
    ROOT / "bench.py",
]

# Names that are files of this repository, not of the reference.
OWN = {"vp_device.cuh", "vp_traverse.cuh", "vp_path.cuh", "vp_internal.h", "volprim_b200.h", "vp_capi.cu",
       "vp_build.cu", "vp_render.cu", "vp_wavefront.cu", "vp_server.cu", "vp_emission.cu", "vp_env.cu",
       "vp_io.cu", "vp_static.cu", "vp_oracle.cpp", "ref_pin.cpp", "bench.py", "api.py", "serving.py",
       "scenes.py", "emission.py", "autograd.py", "oracle.py", "emission_oracle.py", "mitsuba_scene.h",
       "vp_render.cpp", "make_golden.py", "distributed.py", "io.py", "_capi.py", "build_lib.py",
       "__graft_entry__.py", "conftest.py", "validation_scenes.py"}


def _ref_files():
    by_name = {}
    for p in REF.rglob("*"):
        if p.is_file() and ".git" not in p.parts:
            by_name.setdefault(p.name, []).append(p)
    return by_name


def _line_count(p: Path, cache={}) -> int:
    if p not in cache:
        with open(p, "rb") as f:
            cache[p] = sum(1 for _ in f)
    return cache[p]


def _citations():
    for src in SOURCES:
        if not src.is_file():
            continue
        text = src.read_text(errors="replace")
        for m in CITE.finditer(text):
            path, ranges = m.group(1), m.group(2)
            name = path.rsplit("/", 1)[-1]
            if name in OWN or path.startswith(("tests/", "oracle/", "cuda-volprim_b200/", "profiles/")):
                continue
            hi = max(int(x) for x in re.findall(r"\d+", ranges))
            lineno = text.count("\n", 0, m.start()) + 1
            yield src.relative_to(ROOT), lineno, path, hi


@pytest.mark.skipif(not REF.is_dir(), reason="reference tree not present")
def test_reference_citations_resolve():
    by_name = _ref_files()
    bad = []
    n = 0
    for src, lineno, path, hi in _citations():
        name = path.rsplit("/", 1)[-1]
        cands = [p for p in by_name.get(name, []) if p.as_posix().endswith("/" + path.lstrip("./")) or p.name == path]
        n += 1
        if not cands:
            bad.append(f"{src}:{lineno}: {path}:{hi} names no file of the reference")
        elif max(_line_count(p) for p in cands) < hi:
            bad.append(f"{src}:{lineno}: {path}:{hi} is past the end ({max(_line_count(p) for p in cands)} lines)")
    assert n > 100, "the citation scan found too few citations"
    assert not bad, "\n".join(bad)
