"""GPU parity of the directional and point lights' next-event estimates, and of the disk and sphere
lights' analytic geometry (disk_mesh.cu, sphere_mesh.cu): camera rays see the emitters through the
area-light program, shadow rays are blocked by them, and their next-event estimates follow
LightSampler.h.  Checked against the CPU restatement through the C ABI.

Bars: closest-hit index, t and barycentrics and any-hit bit-identical to the oracle's brute-force loop
(triangles, then the emitters in light order, ties to the lower index); images as for the other
scenes (>= 97% of pixels within 1e-3 after 4 frames, relMSE < 1e-3).
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


def test_emitter_geometry_queries_bit_exact():
    data = scenes.analytic_light_scene(16, 16)
    R = sc.Renderer(data)
    O = oc.OracleScene(data)
    rng = np.random.default_rng(5)
    n = 20000
    # rays from random points in the box aimed at random points of the disk and the sphere, plus random rays
    orig = rng.uniform(-0.9, 0.9, (n, 3))
    disk_c, sph_c = np.array([0.0, 0.95, -0.3]), np.array([0.1, 0.1, -0.6])
    tgt = np.where(rng.uniform(size=(n, 1)) < 0.5, disk_c + rng.uniform(-0.25, 0.25, (n, 3)) * [1, 0, 1],
                   sph_c + rng.normal(size=(n, 3)) * 0.05)
    tgt[: n // 4] = rng.uniform(-1, 1, (n // 4, 3))
    d = tgt - orig
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    tmax = np.where(rng.uniform(size=n) < 0.5, 1e27, rng.uniform(0.05, 2.0, n))
    rays = np.concatenate([orig, np.full((n, 1), 1e-4), d, tmax[:, None]], 1).astype(np.float32)
    d_ot = torch.from_numpy(np.ascontiguousarray(rays[:, :4])).cuda()
    d_dt = torch.from_numpy(np.ascontiguousarray(rays[:, 4:])).cuda()
    prim = torch.empty(n, dtype=torch.int32, device="cuda")
    t = torch.empty(n, dtype=torch.float32, device="cuda")
    bary = torch.empty((n, 2), dtype=torch.float32, device="cuda")
    anyh = torch.empty(n, dtype=torch.int32, device="cuda")
    nat.call("pt_trace_closest", R.ctx, d_ot.data_ptr(), d_dt.data_ptr(), n, prim.data_ptr(), t.data_ptr(), bary.data_ptr())
    nat.call("pt_trace_any", R.ctx, d_ot.data_ptr(), d_dt.data_ptr(), n, anyh.data_ptr())
    R.sync()
    bp, bt, bb, ba = O.trace(rays, brute=True)
    gp, gt, gb, ga = prim.cpu().numpy(), t.cpu().numpy(), bary.cpu().numpy(), anyh.cpu().numpy()
    n_tris = len(data.flat_triangles()[0])
    print("emitter hits:", int((bp >= n_tris).sum()), "of", n)
    assert (bp == n_tris).sum() > 1000 and (bp == n_tris + 1).sum() > 1000  # the disk and the sphere are hit
    assert np.array_equal(gp, bp), np.flatnonzero(gp != bp)[:10]
    assert np.array_equal(gt.view(np.uint32), bt.view(np.uint32))
    assert np.array_equal(gb.view(np.uint32), bb.view(np.uint32))
    assert np.array_equal(ga, ba)
    R.close()


def test_disk_and_sphere_light_images_match_the_oracle():
    w = h = 48
    data = scenes.analytic_light_scene(w, h)
    R = sc.Renderer(data)
    R.render(4)
    got = R.readback()
    O = oc.OracleScene(data)
    ref, _ = O.render(0, 4, accum=np.zeros((h, w, 4), np.float32), threads=8)
    assert np.all(np.isfinite(got))
    rel = np.abs(got[..., :3] - ref[..., :3]) / np.maximum(np.abs(ref[..., :3]), 1e-3)
    pix_ok = np.all(rel <= 1e-3, axis=-1).mean()
    print("pixels within 1e-3:", pix_ok, "relMSE", rel_mse(got, ref), "max", float(ref.max()))
    assert pix_ok >= 0.97
    assert rel_mse(got, ref) < 1e-3
    R.close()


def test_directional_and_point_light_images_match_the_oracle():
    """DirectionalLight and PointLight next-event estimation (LightSampler.h:20-37) in an open scene."""
    w = h = 48
    data = scenes.open_lights_scene(w, h)
    assert [type(L).__name__ for L in data.lights] == ["DirectionalLight", "PointLight"]
    R = sc.Renderer(data)
    R.render(4)
    got = R.readback()
    O = oc.OracleScene(data)
    ref, _ = O.render(0, 4, accum=np.zeros((h, w, 4), np.float32), threads=8)
    assert np.all(np.isfinite(got))
    lit = float(np.mean(ref[..., :3].sum(-1) > 0))
    rel = np.abs(got[..., :3] - ref[..., :3]) / np.maximum(np.abs(ref[..., :3]), 1e-3)
    pix_ok = np.all(rel <= 1e-3, axis=-1).mean()
    print("directional + point: pixels within 1e-3:", pix_ok, "relMSE", rel_mse(got, ref), "lit fraction", lit)
    assert lit > 0.3
    assert pix_ok >= 0.97
    assert rel_mse(got, ref) < 1e-3
    R.close()
