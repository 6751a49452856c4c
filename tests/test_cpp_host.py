"""The C++ scene-object classes (include/orf_b200_scene.hpp) through the example host program
open_rendering_framework_b200/render_box: it links and loads the library without a GPU, and on a GPU
its image equals the Python path's on the same scene."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from open_rendering_framework_b200 import scene as sc
from open_rendering_framework_b200 import scenes

BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "open_rendering_framework_b200", "render_box")


def test_example_links_and_reports_usage():
    r = subprocess.run([BIN], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


@pytest.mark.gpu
def test_cpp_classes_render_the_same_image_as_python():
    w = h = 48
    frames = 8
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "img.raw")
        r = subprocess.run([BIN, out, str(w), str(h), str(frames)], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        cpp = np.fromfile(out, np.float32).reshape(h, w, 4)
    bp, bi = scenes.box()
    lp, li = scenes.quad_light((0.0, 0.99, 0.0), 0.25)
    data = sc.SceneData(sc.PathTracer(max_depth=8), sc.PinholeCamera((0, 0, 0.9), (0, 0, -1), (0, 1, 0), 60.0, w, h),
                        sc.ConstantBackground((0, 0, 0)), [sc.Mesh(bp, bi, sc.DiffuseMaterial((0.7, 0.7, 0.7)))],
                        [sc.TriangleAreaLight(lp, li, (15, 15, 15))])
    R = sc.Renderer(data)
    R.render(frames)
    py = R.readback()
    R.close()
    assert np.all(np.isfinite(cpp)) and cpp[..., :3].mean() > 0
    assert np.array_equal(cpp, py)


@pytest.mark.gpu
def test_cpp_classes_render_a_translucent_env_lit_scene_like_python():
    """EnvMapBackground (.hdr), EnvMapLight, TranslucentMaterial (from an OBJ file), RoughDiffuseMaterial,
    PointLight, DirectionalLight, SphericalLight and DiskAreaLight through the C++ classes: the image
    equals the Python path's on the same files, bit for bit."""
    import io_samples

    w, h, frames = 48, 40, 4
    with tempfile.TemporaryDirectory() as d:
        obj = os.path.join(d, "sphere.obj")
        pos, idx, nrm, nidx = scenes.icosphere(3, 0.5)
        with open(obj, "w") as f:
            f.write("".join("v %.7g %.7g %.7g\n" % tuple(p) for p in pos))
            f.write("".join("vn %.7g %.7g %.7g\n" % tuple(n) for n in nrm))
            f.write("".join("f %d//%d %d//%d %d//%d\n" % (a + 1, x + 1, b + 1, y + 1, c + 1, z + 1) for (a, b, c), (x, y, z) in zip(idx, nidx)))
        hdr = os.path.join(d, "sky.hdr")
        sky = scenes.sky_envmap(64, 32, sun_peak=2.0e3, sun_sigma_deg=6.0)
        with open(hdr, "wb") as f:
            f.write(io_samples.hdr_bytes(io_samples.rgbe_from_float(sky[::-1, :, :3]), rle=True))
        out = os.path.join(d, "img.raw")
        r = subprocess.run([BIN, "--translucent", out, obj, hdr, str(w), str(h), str(frames)], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        cpp = np.fromfile(out, np.float32).reshape(h, w, 4)
        skin = sc.TranslucentMaterial()
        floor_mat = sc.RoughDiffuseMaterial(color=(0.5, 0.45, 0.4), roughness=(0.3, 0.3), normal_distribution=sc.GGX_DISTRIBUTION)
        fp_ = np.array([(-3, -0.55, -3), (3, -0.55, -3), (3, -0.55, 3), (-3, -0.55, 3)], np.float32)
        fi = np.array([(0, 2, 1), (0, 3, 2)], np.int32)
        meshes = sc.load_obj(obj, material=skin) + [sc.Mesh(fp_, fi, floor_mat)]
        lights = [sc.EnvMapLight(), sc.PointLight((0.6, 1.5, 0.8), (3.0, 3.0, 3.0)), sc.DirectionalLight((0.0, -1.0, 0.0), (0.5, 0.5, 0.5)),
                  sc.SphericalLight(position=(-0.8, 0.6, 0.3), radiance=(20.0, 15.0, 10.0), radius=0.05),
                  sc.DiskAreaLight(position=(0.5, 1.2, -0.5), radiance=(5.0, 5.0, 5.0), radius=0.2, theta=180.0, phi=0.0)]
        data = sc.SceneData(sc.PathTracer(max_depth=6), sc.PinholeCamera((0.0, 0.35, 2.0), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 36.0, w, h),
                            sc.EnvMapBackground(path=hdr), meshes, lights, probe_samples=64)
        R = sc.Renderer(data)
        R.render(frames)
        py = R.readback()
        st = R.stats()
        R.close()
    assert st.dipole_gathers > 0
    assert np.all(np.isfinite(cpp)) and cpp[..., :3].mean() > 0
    assert np.array_equal(cpp.view(np.uint32), py.view(np.uint32))
