"""GPU parity of the wavefront path tracer against the CPU restatement of the reference's recursive
tracer (oracle/orc/orc_trace.cpp), through the C ABI.

Bars (stated in the tests):
* BVH queries: closest-hit triangle index, t and barycentrics bit-identical to a brute-force loop
  over all triangles with the same Moller-Trumbore test (ties go to the lower index); any-hit
  identical.
* Images: the same camera samples with the same random streams.  A path differs only where a
  last-ulp difference between CUDA's and glibc's transcendentals flips a branch (a Fresnel or
  masking test, a Russian-roulette comparison against a computed probability), so at least 97% of
  pixels agree within 1e-3 relative after 4 frames, and the whole image within relMSE 1e-3.
* Converged images (64 spp) agree within relMSE 2e-3 -- below the 64-spp images' own sample variance
  (relMSE of one half of the frames against the other half, measured in the test).
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


def small_scene(w=32, h=32, model=sc.WALTER_MODEL, rr=0, depth=8):
    return scenes.single_scene(width=w, height=h, metal_subdiv=3, glass_subdiv=2, max_depth=depth, rr_start_depth=rr,
                               metal_model=model, glass_model=model)


def random_rays(n, seed):
    rng = np.random.default_rng(seed)
    o = rng.uniform(-0.95, 0.95, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    tmax = np.where(rng.uniform(size=n) < 0.5, 1e27, rng.uniform(0.05, 1.5, n))
    return np.concatenate([o, np.full((n, 1), 1e-4), d, tmax[:, None]], 1).astype(np.float32)


def test_bvh_closest_and_any_hit_bit_exact():
    data = small_scene()
    R = sc.Renderer(data)
    O = oc.OracleScene(data)
    # random rays inside the box plus rays aimed exactly at triangle vertices and edge midpoints
    rays = random_rays(20000, 1)
    tp, _, _ = data.flat_triangles()
    rng = np.random.default_rng(2)
    pick = rng.integers(0, len(tp), 4000)
    targets = np.concatenate([tp[pick, 0:3], 0.5 * (tp[pick, 3:6] + tp[pick, 6:9])])
    orig = rng.uniform(-0.5, 0.5, (len(targets), 3)).astype(np.float32)
    d = targets - orig
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    extra = np.concatenate([orig, np.full((len(d), 1), 1e-4), d, np.full((len(d), 1), 1e27)], 1).astype(np.float32)
    rays = np.concatenate([rays, extra])
    n = len(rays)
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
    assert (bp >= 0).mean() > 0.5
    assert np.array_equal(gp, bp), np.flatnonzero(gp != bp)[:10]
    assert np.array_equal(gt.view(np.uint32), bt.view(np.uint32))
    assert np.array_equal(gb.view(np.uint32), bb.view(np.uint32))
    assert np.array_equal(ga, ba)
    R.close()


@pytest.mark.parametrize("model", [sc.WALTER_MODEL, sc.VISIBLE_NORMALS_MODEL, sc.MULTISCATTERING_MODEL])
def test_render_matches_cpu_restatement(model):
    w = h = 32
    data = small_scene(w, h, model=model)
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
    print("model", model, "pixels within 1e-3:", pix_ok, "relMSE", rel_mse(got, ref), "segments", st.segments)
    assert pix_ok >= 0.97
    assert rel_mse(got, ref) < 1e-3
    assert np.array_equal(got[..., 3], np.ones((h, w), np.float32))
    R.close()


def test_converged_image_matches_and_is_below_sample_variance():
    w = h = 48
    data = small_scene(w, h)
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


@pytest.mark.parametrize("big", [False, True])
def test_traversal_variants_leave_identical_images(big):
    # the persistent kernels on the 4-wide BVH and on the BVH2, and the one-ray-per-thread kernels,
    # find the same closest hits and occlusions, so the images are bit-identical;
    data = scenes.single_scene(width=24, height=24) if big else small_scene(24, 24)
    imgs = []
    # the material binning is a stable partition, the same for every chunk size (sort granularity);
    # every path's arithmetic is its own, so the overlapped and the in-order schedules, and one or two
    # wavefronts in flight, agree
    for opts in ({}, {"bvh4": 0}, {"extend_mode": 0}, {"bin_items": 4}, {"bin_items": 16}, {"overlap": 0},
                 {"dual": 0}, {"dual": 0, "overlap": 0}):
        R = sc.Renderer(data)
        for k, v in opts.items():
            nat.call("pt_set_option", R.ctx, k.encode(), v)
        R.render(3)
        imgs.append(R.readback())
        R.close()
    for img in imgs[1:]:
        assert np.array_equal(imgs[0].view(np.uint32), img.view(np.uint32))


def test_render_frames_in_one_call_equal_frame_by_frame():
    data = small_scene(16, 16)
    R1 = sc.Renderer(data)
    R1.render(6)
    a = R1.readback()
    R2 = sc.Renderer(data, max_paths_in_flight=16 * 16 * 2)  # forces three passes of two frames
    R2.render(6)
    b = R2.readback()
    R3 = sc.Renderer(data)
    for _ in range(6):
        R3.renderScene()
    c = R3.readback()
    assert np.array_equal(a, b) and np.array_equal(a, c)
    for r in (R1, R2, R3):
        r.close()


@pytest.mark.parametrize("w,h,max_paths", [(1, 1, None), (33, 17, None), (7, 1, 1), (33, 17, 100)])
def test_ragged_sizes_and_tiny_wavefronts_match_oracle(w, h, max_paths):
    """Images whose pixel count is no multiple of a warp or a block, and wavefronts smaller than a frame
    (one chunk per frame then), against the CPU restatement; a render of zero frames changes nothing."""
    data = small_scene(w, h)
    R = sc.Renderer(data, max_paths_in_flight=max_paths)
    R.render(3)
    img = R.readback()
    R.render(0)
    assert np.array_equal(img.view(np.uint32), R.readback().view(np.uint32))
    O = oc.OracleScene(data)
    ref, _ = O.render(0, 3, accum=np.zeros((h, w, 4), np.float32), threads=4)
    rel = np.abs(img[..., :3].astype(np.float64) - ref[..., :3]) / np.maximum(np.abs(ref[..., :3]), 1e-3)
    frac = float(np.mean(np.all(rel <= 1e-3, axis=-1)))
    err = float(np.mean((img[..., :3] - ref[..., :3]) ** 2 / (ref[..., :3].astype(np.float64) ** 2 + 1e-2)))
    print("%dx%d, max paths %s: %.4f of pixels within 1e-3, relMSE %.3e" % (w, h, max_paths, frac, err))
    assert np.all(np.isfinite(img)) and err < 1e-3
    if w * h >= 64:
        assert frac >= 0.95
    R.close()


def test_patch_outside_pixels_are_black_with_unit_alpha():
    data = small_scene(16, 16)
    data.camera.patch_origin = (4, 4)
    data.camera.patch_dims = (5, 5)
    R = sc.Renderer(data)
    R.render(2)
    img = R.readback()
    O = oc.OracleScene(data)
    ref, _ = O.render(0, 2, accum=np.zeros((16, 16, 4), np.float32), threads=4)
    outside = np.ones((16, 16), bool)
    outside[4:10, 4:10] = False   # x, y in [origin, origin + dims] inclusive (path_tracer.cu:36-43)
    assert np.all(img[outside][:, :3] == 0) and np.all(img[outside][:, 3] == 1)
    assert np.all(ref[outside][:, :3] == 0)
    R.close()


def test_invalid_parameters_rejected():
    data = small_scene(8, 8)
    R = sc.Renderer(data)
    bad = sc.RoughTransparentMaterial(ior=-1.0)
    p = bad.params()
    mid = __import__("ctypes").c_uint32()
    assert nat.lib().pt_material_create(R.ctx, bad.type, __import__("ctypes").byref(p), __import__("ctypes").sizeof(p),
                                        __import__("ctypes").byref(mid)) == 1
    assert nat.lib().pt_set_integrator(R.ctx, 5, float("nan"), None, 0) == 1
    assert nat.lib().pt_render_frames(None, 0, 1) == 1
    R.close()


@pytest.mark.gpu
def test_bvh_hits_far_from_origin_bit_exact():
    # the scene shrunk 100x and moved 500 units from the origin: coordinates on a coarse float grid, so
    # many rays have an exactly zero direction component and run exactly inside a box's face plane
    # (the slab tests must not cull those boxes)
    data = small_scene()
    for m in data.meshes:
        m.positions = np.ascontiguousarray(m.positions * np.float32(0.01) + np.float32(500.0), np.float32)
    R = sc.Renderer(data)
    O = oc.OracleScene(data)
    tp, _, _ = data.flat_triangles()
    rng = np.random.default_rng(5)
    n = 8000
    pick = rng.integers(0, len(tp), n)
    w = rng.dirichlet([1, 1, 1], n).astype(np.float32)
    w[: n // 3] = np.array([1, 0, 0], np.float32)
    w[n // 3: 2 * n // 3] = np.array([0.5, 0.5, 0], np.float32)
    targets = tp[pick, 0:3] * w[:, 0:1] + tp[pick, 3:6] * w[:, 1:2] + tp[pick, 6:9] * w[:, 2:3]
    orig = (rng.uniform(-0.9, 0.9, (n, 3)) * 0.01 + 500.0).astype(np.float32)
    orig[::4, 1] = targets[::4, 1]  # a quarter of the rays run in the horizontal plane of their target
    d = (targets - orig).astype(np.float64)
    keep = np.linalg.norm(d, axis=1) > 0
    d, orig = d[keep], orig[keep]
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    n = len(d)
    assert np.mean(np.any(d == 0, axis=1)) > 0.2  # the case under test occurs
    rays = np.concatenate([orig, np.full((n, 1), 1e-6), d, np.full((n, 1), 1e27)], 1).astype(np.float32)
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
    assert (bp >= 0).mean() > 0.5
    assert np.array_equal(prim.cpu().numpy(), bp)
    assert np.array_equal(t.cpu().numpy().view(np.uint32), bt.view(np.uint32))
    assert np.array_equal(bary.cpu().numpy().view(np.uint32), bb.view(np.uint32))
    assert np.array_equal(anyh.cpu().numpy(), ba)
    R.close()
