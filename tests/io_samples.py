"""Sample .hdr and .obj files for the scene-ingestion tests, written from seeded data.

Shared by tests/test_io.py and tests/golden/make_golden_io.py (which records what the reference's own
readers make of them).  The RGBE encoder and the run-length encoder here are written from the Radiance
format description (4 bytes per texel: a shared exponent byte e and mantissas m with value
(m + 0.5) * 2^(e - 136); new-style scanlines: 2, 2, width high, width low, then the four byte planes
as runs (count | 0x80, value) and literal spans (count, bytes)).
"""
import math
import os

import numpy as np


def rgbe_from_float(rgb):
    """float [..., 3] -> uint8 [..., 4] (the usual frexp encoding)."""
    rgb = np.asarray(rgb, np.float64)
    out = np.zeros(rgb.shape[:-1] + (4,), np.uint8)
    m = rgb.max(axis=-1)
    nz = m > 1e-32
    mant, ex = np.frexp(np.where(nz, m, 1.0))
    scale = np.where(nz, mant * 256.0 / np.where(nz, m, 1.0), 0.0)
    out[..., :3] = np.clip(np.floor(rgb * scale[..., None]), 0, 255).astype(np.uint8)
    out[..., 3] = np.where(nz, ex + 128, 0).astype(np.uint8)
    return out


def _rle_plane(plane):
    out = bytearray()
    n = len(plane)
    i = 0
    while i < n:
        j = i + 1
        while j < n and j - i < 127 and plane[j] == plane[i]:
            j += 1
        if j - i >= 4:
            out += bytes([0x80 | (j - i), plane[i]])
            i = j
            continue
        j = i + 1
        while j < n and j - i < 128:
            if j + 3 < n and plane[j] == plane[j + 1] == plane[j + 2] == plane[j + 3]:
                break
            j += 1
        out += bytes([j - i]) + bytes(plane[i:j])
        i = j
    return bytes(out)


def hdr_bytes(rgbe, rle=True, exposure=None, comments=("# written by io_samples",)):
    """A Radiance file for uint8 texels [h, w, 4] (scanline 0 first)."""
    h, w, _ = rgbe.shape
    head = "#?RADIANCE\n" + "".join(c + "\n" for c in comments) + "FORMAT=32-bit_rle_rgbe\n"
    if exposure is not None:
        head += "EXPOSURE=%s\n" % exposure
    head += "\n-Y %d +X %d\n" % (h, w)
    body = bytearray()
    for y in range(h):
        row = rgbe[y]
        if rle and 8 <= w <= 0x7FFF:
            body += bytes([2, 2, w >> 8, w & 0xFF])
            for ch in range(4):
                body += _rle_plane(row[:, ch].tolist())
        else:
            body += row.tobytes()
    return head.encode() + bytes(body)


def hdr_samples():
    """(name, file bytes) of the sample .hdr files."""
    rng = np.random.default_rng(7)
    out = []
    for (w, h, rle, exposure) in ((64, 32, True, None), (300, 20, True, 2.5), (5, 7, False, None), (40, 9, False, 0.5),
                                  (96, 48, True, None)):
        rgb = rng.lognormal(0.0, 2.0, (h, w, 3))
        rgb[rng.uniform(size=(h, w)) < 0.1] = 0.0                      # zero texels (exponent byte 0)
        rgb[:, : w // 3] = rgb[:, :1]                                  # runs for the RLE coder
        out.append(("s_%dx%d_%s_%s.hdr" % (w, h, "rle" if rle else "flat", exposure), hdr_bytes(rgbe_from_float(rgb), rle, exposure)))
    return out


OBJ_SAMPLES = {
    "tri_v.obj": """# plain vertex indices
v 0 0 0
v 1 0 0
v 1 1 0
v 0 1 0
v 0.5 0.5 1
f 1 2 3
f 1 3 4
f 1 2 5 4
""",
    "forms.obj": """v -1 -1 0
v 1 -1 0
v 1 1 0
v -1 1 0
vt 0 0
vt 1 0
vt 1 1
vt 0 1
vn 0 0 1
vn 0 0.6 0.8
g quad_vtn
f 1/1/1 2/2/1 3/3/2 4/4/2
g quad_vt
f 1/1 2/2 3/3 4/4
g quad_vn
f 1//1 2//1 3//2
f 1//2 3//2 4//1
""",
    "groups.obj": """mtllib groups.mtl
v 0 0 0
v 1 0 0
v 1 1 0
v 0 1 0
v 0 0 1
v 1 0 1
usemtl red
f 1 2 3
g wall
f 1 3 4
usemtl blue
f 2 6 3
f 5 6 2 1
g floor
usemtl red
f -1 -2 -3
g empty_group
""",
    "groups.mtl": """newmtl red
Kd 0.8 0.1 0.1
newmtl blue
Ka 0.1 0.1 0.1
Kd 0.1 0.2 0.9
""",
}


def write_samples(directory):
    """Write every sample into `directory`; returns {name: path}."""
    os.makedirs(directory, exist_ok=True)
    paths = {}
    for name, data in hdr_samples():
        p = os.path.join(directory, name)
        with open(p, "wb") as f:
            f.write(data)
        paths[name] = p
    for name, text in OBJ_SAMPLES.items():
        p = os.path.join(directory, name)
        with open(p, "w") as f:
            f.write(text)
        paths[name] = p
    return paths
