"""The .hdr environment path on the device (pt_set_envmap_hdr: RGBE texels uploaded and expanded by a
kernel) against the host decode (pt_hdr_read + pt_set_envmap), and an OBJ model rendered through the
C ABI against the CPU restatement of the reference's tracer.

Bars: environment tables and lookups bit-identical between the two paths (the decode is exact);
the OBJ scene's image as for the other scenes (>= 97% of pixels within 1e-3 after 4 frames,
relMSE < 1e-3).
"""
import os

import numpy as np
import pytest

import io_samples
from oracle import oracle_ctypes as oc
from open_rendering_framework_b200 import _native as nat
from open_rendering_framework_b200 import scene as sc
from open_rendering_framework_b200 import scenes

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def rel_mse(img, ref):
    img = np.asarray(img, np.float64)[..., :3]
    ref = np.asarray(ref, np.float64)[..., :3]
    return float(np.mean((img - ref) ** 2 / (ref ** 2 + 1e-2)))


def env_scene(background, w=16, h=16):
    data = scenes.single_scene(width=w, height=h, metal_subdiv=2, glass_subdiv=1)
    data.background = background
    return data


def test_hdr_device_decode_equals_host_decode(tmp_path):
    paths = io_samples.write_samples(str(tmp_path))
    for name in ("s_300x20_rle_2.5.hdr", "s_96x48_rle_None.hdr", "s_40x9_flat_0.5.hdr"):
        dev = sc.Renderer(env_scene(sc.EnvMapBackground(path=paths[name])))
        host = sc.Renderer(env_scene(sc.EnvMapBackground(rgba=sc.read_hdr(paths[name]))))
        for a, b in zip(dev.envmap_tables(), host.envmap_tables()):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), name
        rng = np.random.default_rng(1)
        d = rng.normal(size=(4096, 3)).astype(np.float32)
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        outs = []
        for R in (dev, host):
            dd = torch.from_numpy(d).cuda()
            looked = torch.empty_like(dd)
            seeds = torch.arange(1, 257, dtype=torch.int32, device="cuda")
            sd = torch.empty((256, 3), dtype=torch.float32, device="cuda")
            sl = torch.empty((256, 3), dtype=torch.float32, device="cuda")
            nat.call("pt_env_query", R.ctx, dd.data_ptr(), 4096, looked.data_ptr(), seeds.data_ptr(), 256, sd.data_ptr(), sl.data_ptr())
            R.sync()
            outs.append([looked.cpu().numpy(), sd.cpu().numpy(), sl.cpu().numpy()])
        for a, b in zip(*outs):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), name
        dev.close()
        host.close()


def test_obj_model_renders_like_the_oracle(tmp_path):
    paths = io_samples.write_samples(str(tmp_path))
    w = h = 40
    # the diffuse box and quad light of the single scene, plus the OBJ's groups (three materials from its
    # material library) scaled into the box
    bp, bi = scenes.box()
    meshes = [sc.Mesh(bp, bi, sc.DiffuseMaterial((0.7, 0.7, 0.7)))]
    for m in sc.load_obj(paths["groups.obj"]):
        m.positions = (m.positions * 0.6 + np.array([-0.3, -0.9, -0.6], np.float32)).astype(np.float32)
        meshes.append(m)
    lp, li = scenes.quad_light((0.0, 0.99, 0.0), 0.25)
    data = sc.SceneData(sc.PathTracer(max_depth=8, scene_epsilon=1e-4),
                        sc.PinholeCamera(eye=(0.0, 0.0, 0.9), lookat=(0.0, 0.0, -1.0), up=(0.0, 1.0, 0.0), vfov=60.0, width=w, height=h),
                        sc.ConstantBackground((0.0, 0.0, 0.0)), meshes, [sc.TriangleAreaLight(lp, li, (15.0, 15.0, 15.0))])
    R = sc.Renderer(data)
    R.render(4)
    got = R.readback()
    O = oc.OracleScene(data)
    ref, _ = O.render(0, 4, accum=np.zeros((h, w, 4), np.float32), threads=8)
    rel = np.abs(got[..., :3] - ref[..., :3]) / np.maximum(np.abs(ref[..., :3]), 1e-3)
    pix_ok = np.all(rel <= 1e-3, axis=-1).mean()
    print("pixels within 1e-3:", pix_ok, "relMSE", rel_mse(got, ref))
    assert pix_ok >= 0.97
    assert rel_mse(got, ref) < 1e-3
    R.close()


def test_checkpoint_resume_is_bit_identical(tmp_path):
    from open_rendering_framework_b200 import jsonscene as js

    data = scenes.single_scene(width=32, height=24, metal_subdiv=2, glass_subdiv=1)
    full = sc.Renderer(data)
    full.render(5)
    ref = full.readback()
    full.close()
    a = sc.Renderer(data)
    a.render(3)
    path = js.save_checkpoint(a, str(tmp_path / "frame.json"), {"note": "saved by the test"})
    a.close()
    b = sc.Renderer(data)
    assert js.load_checkpoint(b, path) == 3
    b.render(2)
    got = b.readback()
    b.close()
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_json_scene_renders_like_the_oracle(tmp_path):
    import json

    from open_rendering_framework_b200 import jsonscene as js

    paths = io_samples.write_samples(str(tmp_path))
    bp, bi = scenes.box()
    with open(tmp_path / "box.obj", "w") as f:
        f.write("".join("v %r %r %r\n" % tuple(map(float, p)) for p in bp) + "".join("f %d %d %d\n" % tuple(t + 1) for t in bi))
    lp, li = scenes.quad_light((0.0, 0.99, 0.0), 0.25)
    with open(tmp_path / "light.obj", "w") as f:
        f.write("".join("v %r %r %r\n" % tuple(map(float, p)) for p in lp) + "".join("f %d %d %d\n" % tuple(t + 1) for t in li))
    doc = {"Integrator": {"type": "PathTracer", "parameters": {"max_depth": 8, "scene_epsilon": 0.0001}},
           "Background": {"type": "ConstantBackground", "parameters": {"background_color": [0, 0, 0]}},
           "Camera": {"type": "PinholeCamera", "parameters": {"eye": [0, 0, 0.9], "lookat": [0, 0, -1], "up": [0, 1, 0], "vfov": 60,
                                                              "width": 40, "height": 40}},
           "Lights": [{"type": "TrianglesAreaLight", "parameters": {"path": "light.obj", "radiance": [15, 15, 15]}},
                      {"type": "PointLight", "parameters": {"position": [0.3, 0.2, -0.5], "radiance": [0.3, 0.2, 0.1]}}],
           "Geometries": [{"type": "obj", "parameters": {"path": "box.obj", "material": {"mtl_name": "diffuse_shader",
                                                                                        "mtl_parameters": {"diffuse_color": [0.7, 0.7, 0.7]}}}},
                          {"type": "obj", "parameters": {"path": os.path.basename(paths["groups.obj"]), "position": [-0.3, -0.9, -0.6],
                                                         "scale": [0.6, 0.6, 0.6], "y_rotation": 30,
                                                         "material": {"mtl_name": "lambertian_interface_shader",
                                                                      "mtl_parameters": {"diffuse_color": [0.8, 0.4, 0.2], "ior": 1.5}}}}]}
    with open(tmp_path / "scene.json", "w") as f:
        json.dump(doc, f)
    data = js.load_json_scene(str(tmp_path / "scene.json")).data
    R = sc.Renderer(data)
    R.render(4)
    got = R.readback()
    O = oc.OracleScene(data)
    ref, _ = O.render(0, 4, accum=np.zeros((40, 40, 4), np.float32), threads=8)
    rel = np.abs(got[..., :3] - ref[..., :3]) / np.maximum(np.abs(ref[..., :3]), 1e-3)
    pix_ok = np.all(rel <= 1e-3, axis=-1).mean()
    print("pixels within 1e-3:", pix_ok, "relMSE", rel_mse(got, ref))
    assert pix_ok >= 0.97
    assert rel_mse(got, ref) < 1e-3
    R.close()
