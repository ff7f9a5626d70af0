"""CPU: asset IO (vp_ply_load / vp_ply_save, vp_hdr_load, vp_exr_save) against files written and
parsed here from the formats' published layouts, with the reference's semantics
(src/thesis/host/utils/io/ply.cpp, hdr.cpp, exr.cpp)."""
import math
import struct

import numpy as np
import pytest

import volprim_b200 as vp
from volprim_b200 import io as vio
from volprim_b200 import scenes

NAMES = ["x", "y", "z", "rot_0", "rot_1", "rot_2", "rot_3", "scale_0", "scale_1", "scale_2",
         "albedo_0", "albedo_1", "albedo_2", "sigma_t_0"]


def sample_rows(n, seed=0):
    rng = np.random.default_rng(seed)
    rows = np.zeros((n, 14))
    rows[:, 0:3] = rng.uniform(-1, 1, (n, 3))
    rows[:, 3:7] = scenes.uniform_quaternions(rng, n) * 1.7  # stored unnormalised
    rows[:, 7:10] = rng.normal(math.log(0.05), 0.3, (n, 3))
    rows[:, 10:13] = rng.uniform(0, 1, (n, 3))
    rows[:, 13] = np.exp(rng.normal(0, 0.5, n))
    return rows


def write_ply(path, rows, fmt="binary_little_endian", types=None, face_first=False, extra=True):
    """A PLY with the 14 properties (+ an unrelated 'nx' and, optionally, a face element with a
    list property before the vertex element)."""
    n = len(rows)
    types = types or ["float"] * 14
    names = NAMES[:]
    cols = [rows[:, k] for k in range(14)]
    if extra:  # an unused property in the middle
        names.insert(3, "nx")
        types = types[:3] + ["double"] + types[3:]
        cols.insert(3, np.full(n, 0.25))
    fmt_code = {"float": "f", "double": "d", "uchar": "B", "int": "i", "short": "h"}
    endian = "<" if fmt == "binary_little_endian" else ">"
    header = ["ply", f"format {fmt} 1.0", "comment written by test_io"]
    faces = [(3, [0, 1, 2]), (4, [1, 2, 3, 4])]
    if face_first:
        header += [f"element face {len(faces)}", "property list uchar int vertex_indices"]
    header += [f"element vertex {n}"] + [f"property {t} {nm}" for t, nm in zip(types, names)]
    if not face_first:
        header += [f"element face {len(faces)}", "property list uchar int vertex_indices"]
    header.append("end_header")
    with open(path, "wb") as f:
        f.write(("\n".join(header) + "\n").encode())

        def write_faces():
            for cnt, idx in faces:
                if fmt == "ascii":
                    f.write((" ".join(str(v) for v in [cnt] + idx) + "\n").encode())
                else:
                    f.write(struct.pack(endian + "B" + "i" * cnt, cnt, *idx))

        if face_first:
            write_faces()
        for r in range(n):
            vals = [c[r] for c in cols]
            if fmt == "ascii":
                f.write((" ".join(repr(float(v)) if t in ("float", "double") else str(int(v))
                                  for v, t in zip(vals, types)) + "\n").encode())
            else:
                f.write(b"".join(struct.pack(endian + fmt_code[t], int(v) if t in ("uchar", "int", "short") else v)
                                 for v, t in zip(vals, types)))
        if not face_first:
            write_faces()


@pytest.mark.parametrize("fmt", ["binary_little_endian", "binary_big_endian", "ascii"])
@pytest.mark.parametrize("face_first", [False, True])
def test_ply_load(tmp_path, fmt, face_first):
    rows = sample_rows(57, seed=1)
    p = tmp_path / "g.ply"
    write_ply(p, rows, fmt=fmt, face_first=face_first)
    g = vio.load_ply(p)
    f32 = rows.astype(np.float32)
    assert g.count == 57 and g.scale_is_log
    assert np.array_equal(g.mean, f32[:, 0:3])
    assert np.array_equal(g.quat_wxyz, f32[:, 3:7])
    assert np.array_equal(g.scale, f32[:, 7:10])
    assert np.array_equal(g.albedo, f32[:, 10:13])
    assert np.array_equal(g.density, f32[:, 13])


def test_ply_mixed_property_types_and_override(tmp_path):
    rows = sample_rows(20, seed=2)
    rows[:, 10:13] = np.round(rows[:, 10:13] * 255)  # albedo stored as uchar in this file
    types = ["double"] * 3 + ["float"] * 7 + ["uchar"] * 3 + ["double"]
    p = tmp_path / "m.ply"
    write_ply(p, rows, types=types)
    g = vio.load_ply(p)
    assert np.array_equal(g.mean, rows[:, 0:3].astype(np.float32))
    assert np.array_equal(g.albedo, rows[:, 10:13].astype(np.float32))
    g2 = vio.load_ply(p, albedo_override=(0.5, 0.25, 1.0))
    assert np.all(g2.albedo == np.array([0.5, 0.25, 1.0], np.float32))
    g3 = vio.load_ply(p, albedo_override=(-1.0, 0.25, 1.0))  # any negative: keep the file's
    assert np.array_equal(g3.albedo, g.albedo)


def test_ply_round_trip_and_scene(tmp_path):
    g = vp.Gaussians(*[a for a in (sample_rows(33, 3)[:, 0:3], sample_rows(33, 3)[:, 7:10],
                                   sample_rows(33, 3)[:, 3:7], sample_rows(33, 3)[:, 13],
                                   sample_rows(33, 3)[:, 10:13])], scale_is_log=True)
    p = tmp_path / "rt.ply"
    vio.save_ply(p, g)
    h = vio.load_ply(p)
    for a, b in ((g.mean, h.mean), (g.scale, h.scale), (g.quat_wxyz, h.quat_wxyz), (g.density, h.density),
                 (g.albedo, h.albedo)):
        assert np.array_equal(np.asarray(a, np.float32), b)


def test_ply_errors(tmp_path):
    rows = sample_rows(4)
    p = tmp_path / "bad.ply"
    write_ply(p, rows, extra=False)
    text = p.read_bytes().replace(b"property float sigma_t_0", b"property float opacity")
    p.write_bytes(text)
    with pytest.raises(vp.VpError, match="missing required property 'sigma_t_0'"):
        vio.load_ply(p)
    with pytest.raises(vp.VpError, match="Failed to open PLY file"):
        vio.load_ply(tmp_path / "none.ply")
    q = tmp_path / "trunc.ply"
    write_ply(q, rows, extra=False)
    q.write_bytes(q.read_bytes()[:-60])
    with pytest.raises(vp.VpError, match="truncated"):
        vio.load_ply(q)


def rgbe_encode(rgb):
    """float RGB -> RGBE bytes (Ward's encoding: shared exponent of the largest component)."""
    m = rgb.max(axis=-1)
    out = np.zeros(rgb.shape[:-1] + (4,), np.uint8)
    nz = m > 1e-32
    mant, ex = np.frexp(m[nz])
    scale = mant * 256.0 / m[nz]
    out[nz, :3] = np.clip(np.floor(rgb[nz] * scale[:, None]), 0, 255).astype(np.uint8)
    out[nz, 3] = (ex + 128).astype(np.uint8)
    return out


def rle_channel(b):
    """Radiance new-RLE encoding of one byte plane: runs (>= 4 repeats) and literals."""
    out = bytearray()
    i, n = 0, len(b)
    while i < n:
        j = i
        while j < n and j - i < 127 and b[j] == b[i]:
            j += 1
        if j - i >= 4:
            out += bytes([128 + (j - i), b[i]])
            i = j
            continue
        k = i
        while k < n and k - i < 128:
            if k + 3 < n and b[k] == b[k + 1] == b[k + 2] == b[k + 3]:
                break
            k += 1
        out += bytes([k - i]) + bytes(b[i:k])
        i = k
    return bytes(out)


def write_hdr(path, rgbe, rle=True, magic=b"#?RADIANCE"):
    H, W, _ = rgbe.shape
    with open(path, "wb") as f:
        f.write(magic + b"\n# test\nFORMAT=32-bit_rle_rgbe\nEXPOSURE=1.0\n\n")
        f.write(f"-Y {H} +X {W}\n".encode())
        for y in range(H):
            if rle:
                f.write(bytes([2, 2, W >> 8, W & 255]))
                for c in range(4):
                    f.write(rle_channel(rgbe[y, :, c].tobytes()))
            else:
                f.write(rgbe[y].tobytes())


def decode_rgbe(rgbe):
    e = rgbe[..., 3].astype(np.int32)
    f = np.where(e > 0, np.ldexp(1.0, e - 136), 0.0).astype(np.float32)
    return rgbe[..., :3].astype(np.float32) * f[..., None]


@pytest.mark.parametrize("rle", [True, False])
def test_hdr_load(tmp_path, rle):
    rng = np.random.default_rng(4)
    W, H = 64, 9
    rgb = np.exp(rng.normal(0, 3, (H, W, 3))).astype(np.float32)
    rgb[2, 10:40] = rgb[2, 10]  # runs for the RLE path
    rgb[5] = 0.0
    rgbe = rgbe_encode(rgb)
    p = tmp_path / "env.hdr"
    write_hdr(p, rgbe, rle=rle, magic=b"#?RADIANCE" if rle else b"#?RGBE")
    img = vio.load_hdr(p)
    assert img.shape == (H, W, 3)
    assert np.array_equal(img, decode_rgbe(rgbe))
    # RGBE keeps 8 mantissa bits of the pixel's largest component (a shared exponent)
    assert np.all(np.abs(img - rgb) <= 2 ** -7 * rgb.max(axis=-1, keepdims=True))


def test_hdr_errors(tmp_path):
    p = tmp_path / "bad.hdr"
    p.write_bytes(b"#?NOTHDR\n\n-Y 1 +X 1\n\x00\x00\x00\x00")
    with pytest.raises(vp.VpError, match="bad magic"):
        vio.load_hdr(p)
    p.write_bytes(b"#?RADIANCE\nFORMAT=32-bit_rle_xyze\n\n-Y 1 +X 1\n\x00\x00\x00\x00")
    with pytest.raises(vp.VpError, match="unsupported"):
        vio.load_hdr(p)
    p.write_bytes(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n+Y 1 +X 1\n\x00\x00\x00\x00")
    with pytest.raises(vp.VpError, match="resolution"):
        vio.load_hdr(p)
    p.write_bytes(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y 2 +X 16\n" + bytes([2, 2, 0, 16, 200, 7]))
    with pytest.raises(vp.VpError, match="corrupt"):
        vio.load_hdr(p)


def read_exr(path):
    """Minimal reader of single-part scanline, uncompressed FLOAT EXR files."""
    data = open(path, "rb").read()
    assert struct.unpack_from("<ii", data, 0) == (20000630, 2)
    pos, attrs = 8, {}
    while data[pos] != 0:
        name_end = data.index(b"\0", pos)
        name = data[pos:name_end].decode()
        type_end = data.index(b"\0", name_end + 1)
        typ = data[name_end + 1:type_end].decode()
        size = struct.unpack_from("<i", data, type_end + 1)[0]
        attrs[name] = (typ, data[type_end + 5:type_end + 5 + size])
        pos = type_end + 5 + size
    pos += 1
    chl = attrs["channels"][1]
    chans, q = [], 0
    while chl[q] != 0:
        e = chl.index(b"\0", q)
        chans.append((chl[q:e].decode(), struct.unpack_from("<i", chl, e + 1)[0]))
        q = e + 1 + 16
    assert attrs["compression"][1] == b"\0"
    x0, y0, x1, y1 = struct.unpack("<iiii", attrs["dataWindow"][1])
    W, H = x1 - x0 + 1, y1 - y0 + 1
    offsets = struct.unpack_from(f"<{H}Q", data, pos)
    img = np.zeros((H, W, len(chans)), np.float32)
    for off in offsets:
        y, size = struct.unpack_from("<ii", data, off)
        assert size == 4 * W * len(chans)
        row = np.frombuffer(data, np.float32, W * len(chans), off + 8).reshape(len(chans), W)
        img[y - y0] = row.T
    return [c for c, _ in chans], [t for _, t in chans], img


@pytest.mark.parametrize("flip", [False, True])
def test_exr_save(tmp_path, flip):
    rng = np.random.default_rng(5)
    rgba = rng.uniform(0, 4, (7, 11, 4)).astype(np.float32)
    p = tmp_path / "out.exr"
    vio.save_exr(p, rgba, flip_vertical=flip)
    names, types, img = read_exr(p)
    assert names == ["B", "G", "R"] and types == [2, 2, 2]
    want = rgba[::-1] if flip else rgba
    assert np.array_equal(img[..., 0], want[..., 2])
    assert np.array_equal(img[..., 1], want[..., 1])
    assert np.array_equal(img[..., 2], want[..., 0])
