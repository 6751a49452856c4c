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
