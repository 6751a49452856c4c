"""The device BVH builder (option "bvh_builder" = 1: LBVH over Morton codes, treelet restructuring
(option "bvh_treelets" rounds), SAH leaves and a device 4-wide collapse, SAH-optimal or greedy by option
"bvh_collapse") against brute force and against the host SAH builder.

Hits are decided by the triangle test alone (closest t, ties to the lower triangle index), so any valid
tree must give bit-identical closest hits (index, t, barycentrics) and any-hit answers to a brute-force
loop, and renders bit-identical to those over the host-built tree.  Checked on the single-scene
configuration's full geometry, a heightfield grid (many equal Morton codes along rows), a scene of
duplicated triangles (equal codes), a scene far from the origin, and scenes small enough for the root
to become a leaf.
"""
import numpy as np
import pytest

from oracle import oracle_ctypes as oc
from open_rendering_framework_b200 import _native as nat
from open_rendering_framework_b200 import scene as sc
from open_rendering_framework_b200 import scenes

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

DEVICE = {"bvh_builder": 1}


def rays_into(data, n, seed, lo=-0.95, hi=0.95):
    """Random rays inside [lo, hi]^3 plus rays aimed at triangle vertices and edge midpoints."""
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    tmax = np.where(rng.uniform(size=n) < 0.5, 1e27, rng.uniform(0.05, 1.5, n))
    rays = np.concatenate([o, np.full((n, 1), 1e-4), d, tmax[:, None]], 1)
    tp, _, _ = data.flat_triangles()
    pick = rng.integers(0, len(tp), n // 4)
    targets = np.concatenate([tp[pick, 0:3], 0.5 * (tp[pick, 3:6] + tp[pick, 6:9])])
    orig = rng.uniform(lo, hi, (len(targets), 3))
    dd = targets - orig
    dd /= np.linalg.norm(dd, axis=1, keepdims=True)
    extra = np.concatenate([orig, np.full((len(dd), 1), 1e-4), dd, np.full((len(dd), 1), 1e27)], 1)
    return np.concatenate([rays, extra]).astype(np.float32)


def gpu_trace(R, rays):
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
    return prim.cpu().numpy(), t.cpu().numpy(), bary.cpu().numpy(), anyh.cpu().numpy()


def assert_same_hits(got, ref):
    gp, gt, gb, ga = got
    bp, bt, bb, ba = ref
    assert np.array_equal(gp, bp), np.flatnonzero(gp != bp)[:10]
    assert np.array_equal(gt.view(np.uint32), bt.view(np.uint32))
    assert np.array_equal(gb.view(np.uint32), bb.view(np.uint32))
    assert np.array_equal(ga, ba)


def duplicated_scene():
    """The small test scene with every icosphere triangle present twice (equal Morton codes)."""
    data = scenes.single_scene(width=16, height=16, metal_subdiv=3, glass_subdiv=2)
    for m in data.meshes[1:3]:
        m.vindex = np.ascontiguousarray(np.concatenate([m.vindex, m.vindex]), np.int32)
        if m.nindex is not None:
            m.nindex = np.ascontiguousarray(np.concatenate([m.nindex, m.nindex]), np.int32)
    return data


def heightfield_scene():
    base = scenes.single_scene(width=16, height=16, metal_subdiv=1, glass_subdiv=1)
    meshes = [m for m in base.meshes if not isinstance(m.material, sc.AreaLightMaterial)]  # the light adds its own
    p, i, n, ni = scenes.heightfield(160, extent=1.8, y0=-0.6, seed=4)
    meshes.append(sc.Mesh(p, i, meshes[0].material, n, ni))
    return sc.SceneData(base.integrator, base.camera, base.background, meshes, base.lights)


@pytest.mark.parametrize("opts", [{"bvh_treelets": 0}, {"bvh_treelets": 2}, {"bvh_treelets": 2, "bvh_collapse": 0}],
                         ids=["lbvh", "treelets", "treelets-greedy-collapse"])
@pytest.mark.parametrize("which", ["single_scene", "heightfield", "duplicated"])
def test_device_bvh_hits_bit_exact_vs_brute_force(which, opts):
    data = {"single_scene": lambda: scenes.single_scene(width=16, height=16), "heightfield": heightfield_scene,
            "duplicated": duplicated_scene}[which]()
    R = sc.Renderer(data, build_options=dict(DEVICE, **opts))
    info = R.build_info()
    print(which, info.as_dict())
    assert info.builder == 1 and info.n_triangles == data.n_triangles
    assert info.wide_nodes > 0 and info.bvh2_depth < 64 and np.isfinite(info.sah_cost)
    rays = rays_into(data, 20000, 3)
    O = oc.OracleScene(data)
    assert_same_hits(gpu_trace(R, rays), O.trace(rays, brute=True))
    R.close()


def test_device_bvh_far_from_origin_bit_exact():
    data = scenes.single_scene(width=16, height=16, metal_subdiv=3, glass_subdiv=2)
    for m in data.meshes:
        m.positions = np.ascontiguousarray(m.positions * np.float32(0.01) + np.float32(500.0), np.float32)
    R = sc.Renderer(data, build_options=DEVICE)
    rays = rays_into(data, 8000, 9, lo=500.0 - 0.0095, hi=500.0 + 0.0095)
    O = oc.OracleScene(data)
    assert_same_hits(gpu_trace(R, rays), O.trace(rays, brute=True))
    R.close()


@pytest.mark.parametrize("n_tris", [2, 3, 9])
def test_device_bvh_tiny_scenes(n_tris):
    # with at most bvh_max_leaf triangles the root of the LBVH can itself become a leaf
    rng = np.random.default_rng(n_tris)
    base = scenes.single_scene(width=8, height=8, metal_subdiv=1, glass_subdiv=1)
    P = rng.uniform(-0.8, 0.8, (3 * n_tris, 3)).astype(np.float32)
    I = np.arange(3 * n_tris, dtype=np.int32).reshape(n_tris, 3)
    data = sc.SceneData(base.integrator, base.camera, base.background, [sc.Mesh(P, I, base.meshes[1].material)], [])
    R = sc.Renderer(data, build_options=dict(DEVICE, bvh_max_leaf=15))
    assert R.build_info().builder == 1
    rays = rays_into(data, 4000, n_tris)
    O = oc.OracleScene(data)
    assert_same_hits(gpu_trace(R, rays), O.trace(rays, brute=True))
    R.close()


def test_treelet_restructuring_lowers_the_sah_cost():
    """Rounds of treelet restructuring lower the SAH cost of the device tree on the single-scene
    configuration's geometry, toward the host binned-SAH tree's."""
    data = scenes.single_scene(width=16, height=16)
    costs = {}
    for rounds in (0, 1, 2, 3):
        R = sc.Renderer(data, build_options=dict(DEVICE, bvh_treelets=rounds))
        info = R.build_info()
        assert info.builder == 1
        costs[rounds] = info.sah_cost
        R.close()
    R = sc.Renderer(data)
    host = R.build_info().sah_cost
    R.close()
    print("SAH cost by treelet rounds:", costs, "host binned SAH:", host)
    assert costs[1] < costs[0] and costs[2] <= costs[1] * 1.001 and costs[3] <= costs[2] * 1.001


@pytest.mark.parametrize("which", ["single_scene", "translucent"])
def test_renders_over_device_bvh_equal_host_bvh(which):
    if which == "single_scene":
        data = scenes.single_scene(width=48, height=48)
    else:
        data = scenes.translucent_box_scene(32, 32, probe_samples=64)
    imgs, infos = [], []
    for opts in ({}, DEVICE):
        R = sc.Renderer(data, build_options=opts)
        R.render(3)
        imgs.append(R.readback())
        infos.append(R.build_info().as_dict())
        R.close()
    print(which, "host:", infos[0], "device:", infos[1])
    assert infos[0]["builder"] == 0 and infos[1]["builder"] == 1
    assert np.array_equal(imgs[0].view(np.uint32), imgs[1].view(np.uint32))


def test_rebuild_switches_builder_and_keeps_images():
    data = scenes.single_scene(width=24, height=24, metal_subdiv=4, glass_subdiv=3)
    R = sc.Renderer(data)
    R.render(2)
    a = R.readback()
    R.rebuild(bvh_builder=1)
    R.apply_camera()
    R.frame = 0
    R.render(2)
    b = R.readback()
    assert R.build_info().builder == 1
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert nat.lib().pt_set_option(R.ctx, b"bvh_builder", 2) == 1
    R.close()
