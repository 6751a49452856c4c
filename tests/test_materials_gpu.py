"""GPU parity of the remaining material programs -- smooth glass (transparent_shader.cu), a Lambertian
base under a smooth interface (lambertian_interface_shader.cu) and under a rough interface
(rough_diffuse_shader.cu, Walter / visible-normal / multiscattering models, both distributions) --
against the CPU restatement of the reference's recursive tracer (oracle/orc/orc_trace.cpp), through
the C ABI.

Bars, as for the other materials: the same camera samples consume the same random streams, so at least
97% of pixels agree within 1e-3 relative after 4 frames and the image within relMSE 1e-3; a 64-frame
render agrees within relMSE 2e-3 and below the image's own sample variance (one half of the frames
against the other).
"""
import numpy as np
import pytest

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


@pytest.mark.parametrize("model,dist", [(sc.WALTER_MODEL, sc.BECKMANN_DISTRIBUTION), (sc.VISIBLE_NORMALS_MODEL, sc.GGX_DISTRIBUTION),
                                        (sc.MULTISCATTERING_MODEL, sc.GGX_DISTRIBUTION),
                                        (sc.MULTISCATTERING_MODEL, sc.BECKMANN_DISTRIBUTION)])
def test_layered_and_smooth_glass_images_match_the_oracle(model, dist):
    w = h = 48
    data = scenes.layered_scene(w, h, rough_model=model, rough_distribution=dist)
    R = sc.Renderer(data)
    R.render(4)
    got = R.readback()
    st = R.stats()
    O = oc.OracleScene(data)
    ref, _ = O.render(0, 4, accum=np.zeros((h, w, 4), np.float32), threads=8)
    assert np.all(np.isfinite(got))
    assert st.path_samples == w * h * 4 and st.segments > w * h * 4
    rel = np.abs(got[..., :3] - ref[..., :3]) / np.maximum(np.abs(ref[..., :3]), 1e-3)
    pix_ok = np.all(rel <= 1e-3, axis=-1).mean()
    print("model", model, "dist", dist, "pixels within 1e-3:", pix_ok, "relMSE", rel_mse(got, ref), "capped", st.capped_walks)
    assert pix_ok >= 0.97
    assert rel_mse(got, ref) < 1e-3
    R.close()


def test_layered_converged_image_is_below_sample_variance():
    w = h = 40
    data = scenes.layered_scene(w, h, rough_model=sc.VISIBLE_NORMALS_MODEL, rough_distribution=sc.GGX_DISTRIBUTION)
    R = sc.Renderer(data)
    R.render(64)
    got = R.readback()
    O = oc.OracleScene(data)
    ref, pr = O.render(0, 64, accum=np.zeros((h, w, 4), np.float32), path_radiance=True, threads=8)
    a = pr[:32].mean(axis=0).reshape(h, w, 3)
    b = pr[32:].mean(axis=0).reshape(h, w, 3)
    half_var = rel_mse(a, b)
    err = rel_mse(got, ref)
    print("converged relMSE gpu vs cpu:", err, "half-vs-half relMSE:", half_var)
    assert err < 2e-3
    assert err < half_var
    R.close()


def test_layered_materials_are_rejected_by_the_adjoint():
    data = scenes.layered_scene(16, 16)
    R = sc.Renderer(data)
    nat.call("pt_set_option", R.ctx, b"differentiable", 1)
    R.render(1)
    g = torch.zeros((16, 16, 4), dtype=torch.float32, device="cuda")
    with pytest.raises(nat.PtError) as e:
        nat.call("pt_render_adjoint", R.ctx, 0, 1, g.data_ptr())
    assert e.value.status == 1
    R.close()
