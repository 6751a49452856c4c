"""The scene readers behind the C ABI (pt_hdr_read, pt_obj_*), pinned to the reference's own readers.

tests/golden/ref_io.npz holds what the reference's HDRLoader.cpp (with loadHDRTexture) and glm.cpp,
compiled for the host, make of the sample files of tests/io_samples.py and of the reference's own
data/CedarCity.hdr and data/Plane.obj (tests/golden/make_golden_io.py).  Bars: .hdr texels (RGB)
bit-identical; .obj arrays, counts and group order identical.  Where the compiled reference and its
data are present the readers are also compared with it directly.  These tests need no GPU.
"""
import ctypes
import hashlib
import math
import os

import numpy as np
import pytest

import io_samples
from open_rendering_framework_b200 import _native as nat
from open_rendering_framework_b200 import scene as sc

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = np.load(os.path.join(HERE, "golden", "ref_io.npz"))
# the reference checkout (its data/ and scenes/ folders), named by the ORF_REFERENCE environment
# variable; the tests that read it directly are skipped when it is unset or absent
REF_ROOT = os.environ.get("ORF_REFERENCE", "")
REF_DATA = os.path.join(REF_ROOT, "data") if REF_ROOT else ""


@pytest.fixture(scope="module")
def samples(tmp_path_factory):
    return io_samples.write_samples(str(tmp_path_factory.mktemp("io")))


def obj_arrays(path):
    obj = ctypes.c_void_p()
    nat.call("pt_obj_read", os.fsencode(path), ctypes.byref(obj))
    info = (ctypes.c_uint32 * 5)()
    nat.call("pt_obj_get_info", obj, info)
    nv, nn, nt, ntri, ng = list(info)
    a = {"counts": np.array(list(info), np.uint32), "positions": np.zeros(3 * nv, np.float32), "normals": np.zeros(3 * nn, np.float32),
         "texcoords": np.zeros(2 * nt, np.float32), "vindex": np.zeros(3 * ntri, np.int32), "nindex": np.zeros(3 * ntri, np.int32),
         "tindex": np.zeros(3 * ntri, np.int32), "group": np.zeros(ntri, np.uint32)}
    nat.call("pt_obj_get_arrays", obj, *[a[k].ctypes.data if a[k].size else None for k in
                                          ("positions", "normals", "texcoords", "vindex", "nindex", "tindex", "group")])
    names = []
    for k in range(ng):
        g = sc.ObjGroup()
        nat.call("pt_obj_get_group", obj, k, ctypes.byref(g))
        names.append(g.name.decode())
    nat.call("pt_obj_free", obj)
    a["group_names"] = np.array(names)
    return a


def test_hdr_samples_match_the_reference_reader(samples):
    for name, path in samples.items():
        if not name.endswith(".hdr"):
            continue
        got = sc.read_hdr(path)
        ref = GOLD["hdr/" + name]
        assert got.shape[:2] == ref.shape[:2], name
        assert np.array_equal(got[..., :3].view(np.uint32), ref.view(np.uint32)), name
        assert np.all(got[..., 3] == 1.0)


def test_cedar_city_matches_the_reference_reader():
    path = os.path.join(REF_DATA, "CedarCity.hdr") if REF_DATA else ""
    if not path or not os.path.exists(path):
        pytest.skip("the reference's data/CedarCity.hdr is not present (its digest is pinned in ref_io.npz)")
    got = np.ascontiguousarray(sc.read_hdr(path)[..., :3])
    assert got.shape == tuple(GOLD["cedar/shape"])
    assert np.array_equal(got.reshape(-1, 3)[GOLD["cedar/sample_idx"]].view(np.uint32), GOLD["cedar/sample_rgb"].view(np.uint32))
    assert hashlib.sha256(got.tobytes()).hexdigest() == str(GOLD["cedar/sha256"])


def test_obj_samples_match_the_reference_reader(samples):
    cases = [(n, p) for n, p in samples.items() if n.endswith(".obj")]
    if REF_DATA and os.path.exists(os.path.join(REF_DATA, "Plane.obj")):
        cases.append(("Plane.obj", os.path.join(REF_DATA, "Plane.obj")))
    for name, path in cases:
        got = obj_arrays(path)
        for k in ("counts", "positions", "normals", "texcoords", "vindex", "nindex", "tindex", "group"):
            ref = GOLD["obj/%s/%s" % (name, k)]
            assert np.array_equal(got[k], ref), (name, k)
        assert list(got["group_names"]) == list(GOLD["obj/%s/group_names" % name]), name


def test_live_reference_readers_agree(samples):
    lib = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libref_io.so")
    if not os.path.exists(lib):
        pytest.skip("oracle/_ref/libref_io.so is not built")
    L = ctypes.CDLL(lib)
    for name, path in samples.items():
        if name.endswith(".hdr"):
            w, h = ctypes.c_uint(), ctypes.c_uint()
            L.ref_hdr_load(path.encode(), None, ctypes.c_ulong(0), ctypes.byref(w), ctypes.byref(h))
            buf = np.zeros(4 * w.value * h.value, np.float32)
            L.ref_hdr_load(path.encode(), buf.ctypes.data_as(ctypes.c_void_p), ctypes.c_ulong(buf.size), ctypes.byref(w), ctypes.byref(h))
            assert np.array_equal(buf.reshape(h.value, w.value, 4)[..., :3].view(np.uint32), sc.read_hdr(path)[..., :3].view(np.uint32))


def test_obj_groups_become_meshes_with_their_materials(samples):
    meshes = sc.load_obj(samples["groups.obj"])
    assert [len(m.vindex) for m in meshes] == [1, 3, 1, 1]
    assert meshes[0].material.color == pytest.approx((0.8, 0.1, 0.1))
    assert meshes[1].material.color == pytest.approx((0.1, 0.2, 0.9))
    metal = sc.MetallicMaterial()
    meshes = sc.load_obj(samples["groups.obj"], materials={"blue": metal})
    assert meshes[1].material is metal


@pytest.mark.parametrize("text", [b"#?RGBE\n\n-Y 2 +X 2\n", b"#?RADIANCE\nFORMAT=32-bit_rle_xyze\n\n-Y 2 +X 2\n",
                                  b"#?RADIANCE\n\n+Y 2 +X 2\n" + bytes(16), b"#?RADIANCE\n\n-Y 4 +X 4\n" + bytes(20),
                                  b"#?RADIANCE\nEXPOSURE=0\n\n-Y 1 +X 1\n" + bytes(4)])
def test_bad_hdr_files_are_rejected(tmp_path, text):
    p = tmp_path / "bad.hdr"
    p.write_bytes(text)
    w, h = ctypes.c_uint32(), ctypes.c_uint32()
    with pytest.raises(nat.PtError) as e:
        nat.call("pt_hdr_read", os.fsencode(p), None, 0, ctypes.byref(w), ctypes.byref(h))
    assert e.value.status == 1


@pytest.mark.parametrize("text", ["v 0 0 0\nv 1 0 0\nf 1 2\n", "v 0 0 0\nf 1 2 3\n", "v 0 0\n", "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1//4 2//4 3//4\n"])
def test_bad_obj_files_are_rejected(tmp_path, text):
    p = tmp_path / "bad.obj"
    p.write_text(text)
    obj = ctypes.c_void_p()
    with pytest.raises(nat.PtError) as e:
        nat.call("pt_obj_read", os.fsencode(p), ctypes.byref(obj))
    assert e.value.status == 1


# ---------------------------------------------------------------- JSON scenes (OptixSceneLoader)
from open_rendering_framework_b200 import jsonscene as js  # noqa: E402


def write_json_scene(directory, samples):
    import json
    import shutil

    for name in ("groups.obj", "groups.mtl", "tri_v.obj"):
        shutil.copy(samples[name], os.path.join(directory, name))
    doc = {
        "Integrator": {"type": "PathTracer", "parameters": {"max_depth": 6, "scene_epsilon": 0.0001, "exception_color": [1, 0, 1]}},
        "Background": {"type": "ConstantBackground", "parameters": {"background_color": [0.1, 0.2, 0.3]}},
        "Camera": {"type": "PinholeCamera", "parameters": {"eye": [0, 0.5, 3], "lookat": [0, 0.3, 0], "up": [0, 1, 0], "vfov": 45,
                                                           "width": 40, "height": 32}},
        "Lights": [{"type": "PointLight", "parameters": {"radiance": [2, 2, 2], "position": [0, 2, 1]}},
                   {"type": "DiskAreaLight", "parameters": {"radiance": [3, 3, 3], "position": [0, 2, 0], "radius": 0.3, "theta": 180, "phi": 0}},
                   {"type": "TrianglesAreaLight", "parameters": {"path": "tri_v.obj", "radiance": [1, 1, 1], "position": [0, 3, 0],
                                                                "scale": [0.2, 0.2, 0.2]}}],
        "Geometries": [
            {"type": "obj", "parameters": {"path": "groups.obj", "position": [0, 0, 0], "scale": [1, 1, 1],
                                           "material": {"mtl_name": "rough_diffuse_shader",
                                                        "mtl_parameters": {"diffuse_color": [0.5, 0.4, 0.3], "ior": 1.4, "roughness": [0.2, 0.2],
                                                                           "microfacet_model": 1, "normal_distribution": 1}}}},
            {"type": "obj", "parameters": {"path": "groups.obj", "position": [1, 0, 0], "scale": [2, 1, 1], "rotation": [90, 0, 1, 0],
                                           "y_rotation": 10,
                                           "material": {"mtl_name": "metallic_shader",
                                                        "mtl_parameters": {"real_ior": [0.2, 0.55, 0.9], "imaginary_ior": [3.9, 3.15, 2.4],
                                                                           "roughness": [0.3, 0.3]}}}}],
    }
    path = os.path.join(directory, "scene.json")
    with open(path, "w") as f:
        json.dump(doc, f)
    return path


def test_json_scene_is_read_with_the_reference_schema(tmp_path, samples):
    path = write_json_scene(str(tmp_path), samples)
    S = js.load_json_scene(path)
    d = S.data
    assert d.integrator.max_depth == 6 and d.camera.width == 40 and d.camera.height == 32
    assert d.background.background_color == (0.1, 0.2, 0.3)
    assert [type(L).__name__ for L in d.lights] == ["PointLight", "DiskAreaLight", "TriangleAreaLight"]
    kinds = [type(m.material).__name__ for m in d.meshes]
    assert kinds.count("RoughDiffuseMaterial") == 4 and kinds.count("MetallicMaterial") == 4 and kinds.count("AreaLightMaterial") == 1
    assert d.meshes[0].material.roughness == (0.2, 0.2) and d.meshes[4].material.ior[0] == (0.2, 3.9)
    # the second copy: M = T(1,0,0) Ry(10) R(90 about y) S(2,1,1); vertex (1,0,0) -> x-scaled, rotated by 100 degrees about y
    A, t = js.geometry_transform({"position": [1, 0, 0], "scale": [2, 1, 1], "rotation": [90, 0, 1, 0], "y_rotation": 10})
    v = A @ np.array([1.0, 0.0, 0.0]) + t
    assert v == pytest.approx([1 + 2 * math.cos(math.radians(100)), 0.0, -2 * math.sin(math.radians(100))], abs=1e-6)
    assert S.frame_count == 0 and S.buffer_path is None


def test_reference_scene_file_is_read(tmp_path, samples):
    ref = os.path.join(REF_ROOT, "scenes", "jsonscene.json") if REF_ROOT else ""
    if not ref or not os.path.exists(ref):
        pytest.skip("the reference's scenes/jsonscene.json is not present")
    import json
    import shutil

    # its OBJ files and .hdr are not part of the reference snapshot: stand-ins under the same relative names
    doc = json.load(open(ref))
    for g in doc["Geometries"]:
        p = tmp_path / g["parameters"]["path"]
        p.parent.mkdir(parents=True, exist_ok=True)
        shutil.copy(samples["forms.obj"], p)
    hdr = tmp_path / doc["Background"]["parameters"]["path"]
    hdr.parent.mkdir(parents=True, exist_ok=True)
    shutil.copy(samples["s_64x32_rle_None.hdr"], hdr)
    S = js.load_json_scene(ref, base_dir=str(tmp_path), unsupported_material=sc.DiffuseMaterial((0.2, 0.8, 0.5)))
    d = S.data
    assert d.integrator.max_depth == 100 and (d.camera.width, d.camera.height) == (1200, 1000)
    assert isinstance(d.background, sc.EnvMapBackground) and d.background.rgba.shape == (32, 64, 4)
    assert [type(L).__name__ for L in d.lights] == ["PointLight", "PointLight", "DirectionalLight"]
    assert d.meshes[0].material.color == (1.0, 0.3, 0.7)
    with pytest.raises(ValueError):
        js.load_json_scene(ref, base_dir=str(tmp_path))  # its second geometry uses normal_shader
