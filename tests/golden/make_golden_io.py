"""Generate tests/golden/ref_io.npz from the reference's own scene readers.

oracle/_ref/libref_io.so is the reference's HDRLoader.cpp (with loadHDRTexture) and glm.cpp compiled
for the host by oracle/Makefile.  It reads the sample files of tests/io_samples.py and the reference's
own data/CedarCity.hdr and data/Plane.obj; what it returns is recorded here (the .hdr texels as RGB
float32 -- the reference leaves the fourth channel undefined -- and the .obj arrays as ObjLoader
flattens them).  Run from the repository root:  python tests/golden/make_golden_io.py
(ORF_REFERENCE names the reference checkout whose data/ folder is read).
"""
import ctypes
import hashlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(HERE))
import io_samples  # noqa: E402

REF_IO = os.path.join(ROOT, "oracle", "_ref", "libref_io.so")
REF_DATA = os.path.join(os.environ.get("ORF_REFERENCE", "/root/reference"), "data")
OUT = os.path.join(HERE, "ref_io.npz")


def vp(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def ref_hdr(L, path):
    w, h = ctypes.c_uint(), ctypes.c_uint()
    if not L.ref_hdr_load(path.encode(), None, ctypes.c_ulong(0), ctypes.byref(w), ctypes.byref(h)):
        raise RuntimeError("reference failed on " + path)
    buf = np.zeros(4 * w.value * h.value, np.float32)
    L.ref_hdr_load(path.encode(), vp(buf), ctypes.c_ulong(buf.size), ctypes.byref(w), ctypes.byref(h))
    return buf.reshape(h.value, w.value, 4)[..., :3].copy()


def ref_obj(L, path):
    counts = (ctypes.c_uint * 5)()
    if not L.ref_obj_load(path.encode(), counts, *([None] * 8), 0):
        raise RuntimeError("reference failed on " + path)
    nv, nn, nt, ntri, ng = list(counts)
    a = {"counts": np.array(list(counts), np.uint32), "positions": np.zeros(3 * nv, np.float32), "normals": np.zeros(3 * nn, np.float32),
         "texcoords": np.zeros(2 * nt, np.float32), "vindex": np.zeros(3 * ntri, np.int32), "nindex": np.zeros(3 * ntri, np.int32),
         "tindex": np.zeros(3 * ntri, np.int32), "group": np.zeros(ntri, np.uint32)}
    names = ctypes.create_string_buffer(128 * max(ng, 1))
    L.ref_obj_load(path.encode(), counts, vp(a["positions"]), vp(a["normals"]) if nn else None, vp(a["texcoords"]) if nt else None,
                   vp(a["vindex"]), vp(a["nindex"]), vp(a["tindex"]), vp(a["group"]), names, 128)
    a["group_names"] = np.array([names.raw[128 * k:128 * (k + 1)].split(b"\0")[0].decode() for k in range(ng)])
    return a


def main():
    if not os.path.exists(REF_IO):
        raise SystemExit("oracle/_ref/libref_io.so is not built (needs the reference sources)")
    L = ctypes.CDLL(REF_IO)
    g = {}
    with tempfile.TemporaryDirectory() as d:
        paths = io_samples.write_samples(d)
        for name, p in paths.items():
            if name.endswith(".hdr"):
                g["hdr/" + name] = ref_hdr(L, p)
            elif name.endswith(".obj"):
                for k, v in ref_obj(L, p).items():
                    g["obj/%s/%s" % (name, k)] = v
    cedar = ref_hdr(L, os.path.join(REF_DATA, "CedarCity.hdr"))
    g["cedar/shape"] = np.array(cedar.shape, np.int64)
    g["cedar/sha256"] = np.array(hashlib.sha256(np.ascontiguousarray(cedar).tobytes()).hexdigest())
    rng = np.random.default_rng(3)
    idx = rng.integers(0, cedar.shape[0] * cedar.shape[1], 512)
    g["cedar/sample_idx"] = idx
    g["cedar/sample_rgb"] = cedar.reshape(-1, 3)[idx]
    for k, v in ref_obj(L, os.path.join(REF_DATA, "Plane.obj")).items():
        g["obj/Plane.obj/%s" % k] = v
    np.savez_compressed(OUT, **g)
    print("wrote", OUT, len(g), "arrays")


if __name__ == "__main__":
    main()
