"""The product's BVH builders and traversals (pt_bvh.cu, pt_scene.cuh: stackless BVH2, its short-stack
variant, the 4- and 8-wide BVHs with their ring-and-spill stack), compiled for the host by
tests/native/host_trace.cu, against the brute-force oracle: closest-hit index, t and barycentrics and
any-hit bit-identical, including rays aimed exactly at vertices and edges.  Runs without a GPU (the
same code runs on the device in tests/test_render_gpu.py)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle_ctypes as oc
from open_rendering_framework_b200 import scenes

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "native", "_build", "libhost_trace_w%d.so")
SRC = [os.path.join(HERE, "native", "host_trace.cu"),
       os.path.join(HERE, "..", "open_rendering_framework_b200", "csrc", "pt_bvh.cu")]
HDR = [os.path.join(HERE, "..", "open_rendering_framework_b200", "csrc", f) for f in ("pt_scene.cuh", "pt_math.cuh", "pt_bvh.h")]


@pytest.fixture(scope="module", params=[4, 8], ids=["bvh4", "bvh8"])
def host_lib(request):
    # the wide BVH compiled at both widths (PT_BVH_WIDE), whichever the library uses
    width = request.param
    so = SO % width
    newest = max(os.path.getmtime(p) for p in SRC + HDR)
    if not os.path.exists(so) or os.path.getmtime(so) < newest:
        os.makedirs(os.path.dirname(so), exist_ok=True)
        subprocess.run(["/usr/local/cuda/bin/nvcc", "-std=c++17", "-O2", "--fmad=false", "-Wno-deprecated-gpu-targets",
                        "-DPT_BVH_WIDE=%d" % width, "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-shared"]
                       + SRC + ["-o", so], check=True)
    L = ctypes.CDLL(so)
    L.ht_build.restype = ctypes.c_void_p
    L.ht_build.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_void_p]
    L.ht_free.argtypes = [ctypes.c_void_p]
    L.ht_trace.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long] + [ctypes.c_void_p] * 4
    L.ht_trace_stack.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long] + [ctypes.c_void_p] * 4
    L.ht_trace4.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long] + [ctypes.c_void_p] * 5
    L.ht_build_collapse.restype = ctypes.c_void_p
    L.ht_build_collapse.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_int, ctypes.c_float, ctypes.c_void_p]
    L.ht_from_arrays.restype = ctypes.c_void_p
    L.ht_from_arrays.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint,
                                 ctypes.c_void_p]
    return L


def edge_and_random_rays(tp, n, seed):
    rng = np.random.default_rng(seed)
    pick = rng.integers(0, len(tp), n)
    w = rng.dirichlet([1, 1, 1], n).astype(np.float32)
    w[: n // 3] = np.array([1, 0, 0], np.float32)           # vertices
    w[n // 3: 2 * n // 3] = np.array([0.5, 0.5, 0], np.float32)  # edge midpoints
    targets = tp[pick, 0:3] * w[:, 0:1] + tp[pick, 3:6] * w[:, 1:2] + tp[pick, 6:9] * w[:, 2:3]
    orig = rng.uniform(-0.9, 0.9, (n, 3)).astype(np.float32)
    d = targets - orig
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    tmax = np.where(rng.uniform(size=n) < 0.7, 1e27, rng.uniform(0.05, 2.0, n))
    return np.ascontiguousarray(np.concatenate([orig, np.full((n, 1), 1e-4), d, tmax[:, None]], 1).astype(np.float32))


@pytest.mark.parametrize("subdiv", [(1, 0), (3, 2), (4, 3)])
def test_host_traversal_matches_brute_force(host_lib, subdiv):
    data = scenes.single_scene(width=8, height=8, metal_subdiv=subdiv[0], glass_subdiv=subdiv[1])
    tp, _, _ = data.flat_triangles()
    depth = ctypes.c_int()
    h = host_lib.ht_build(oc.fp(tp), len(tp), ctypes.byref(depth))
    assert h and 0 < depth.value < 64
    rays = edge_and_random_rays(tp, 6000, 11)
    n = len(rays)
    prim, t = np.empty(n, np.int32), np.empty(n, np.float32)
    bary, anyh = np.empty((n, 2), np.float32), np.empty(n, np.int32)
    host_lib.ht_trace(h, oc.fp(rays), n, oc.fp(prim), oc.fp(t), oc.fp(bary), oc.fp(anyh))
    # the short-stack variant of the persistent kernels
    prim2, t2 = np.empty(n, np.int32), np.empty(n, np.float32)
    bary2, anyh2 = np.empty((n, 2), np.float32), np.empty(n, np.int32)
    host_lib.ht_trace_stack(h, oc.fp(rays), n, oc.fp(prim2), oc.fp(t2), oc.fp(bary2), oc.fp(anyh2))
    # the 4-wide BVH of the persistent kernels
    prim4, t4 = np.empty(n, np.int32), np.empty(n, np.float32)
    bary4, anyh4 = np.empty((n, 2), np.float32), np.empty(n, np.int32)
    max_sp = ctypes.c_int()
    assert host_lib.ht_trace4(h, oc.fp(rays), n, oc.fp(prim4), oc.fp(t4), oc.fp(bary4), oc.fp(anyh4), ctypes.byref(max_sp)) == 0
    host_lib.ht_free(h)
    if subdiv == (4, 3):
        assert max_sp.value > 8  # the shared-memory ring overflowed into the spill array
    bp, bt, bb, ba = oc.OracleScene(data).trace(rays, brute=True)
    for p_, t_, b_, a_ in ((prim, t, bary, anyh), (prim2, t2, bary2, anyh2), (prim4, t4, bary4, anyh4)):
        assert np.array_equal(p_, bp)
        assert np.array_equal(t_.view(np.uint32), bt.view(np.uint32))
        assert np.array_equal(b_.view(np.uint32), bb.view(np.uint32))
        assert np.array_equal(a_, ba)


@pytest.mark.parametrize("wide_cost", [0.5, 1.5, 4.0])
def test_sah_optimal_collapse_matches_brute_force(host_lib, wide_cost):
    """The 4-wide tree of the SAH-optimal collapse (option bvh_collapse = 1) over the same BVH2: hits
    bit-exact against brute force, every wide node with at least two children, all triangles reachable."""
    data = scenes.single_scene(width=8, height=8, metal_subdiv=4, glass_subdiv=3)
    tp, _, _ = data.flat_triangles()
    nw = ctypes.c_uint()
    h = host_lib.ht_build_collapse(oc.fp(tp), len(tp), 1, wide_cost, ctypes.byref(nw))
    g = host_lib.ht_build_collapse(oc.fp(tp), len(tp), 0, wide_cost, None)
    assert h and g and nw.value > 0
    rays = edge_and_random_rays(tp, 6000, 5)
    n = len(rays)
    bp, bt, bb, ba = oc.OracleScene(data).trace(rays, brute=True)
    for hh in (h, g):
        prim4, t4 = np.empty(n, np.int32), np.empty(n, np.float32)
        bary4, anyh4 = np.empty((n, 2), np.float32), np.empty(n, np.int32)
        max_sp = ctypes.c_int()
        assert host_lib.ht_trace4(hh, oc.fp(rays), n, oc.fp(prim4), oc.fp(t4), oc.fp(bary4), oc.fp(anyh4), ctypes.byref(max_sp)) == 0
        assert np.array_equal(prim4, bp)
        assert np.array_equal(t4.view(np.uint32), bt.view(np.uint32))
        assert np.array_equal(bary4.view(np.uint32), bb.view(np.uint32))
        assert np.array_equal(anyh4, ba)
        host_lib.ht_free(hh)


def test_single_triangle_and_degenerate_scenes(host_lib):
    # one triangle (root with an empty second child), and many coincident triangles (no centroid split)
    one = np.array([[0, 0, 0, 1, 0, 0, 0, 1, 0]], np.float32)
    same = np.repeat(one, 40, axis=0)
    for tp in (one, same):
        h = host_lib.ht_build(oc.fp(tp), len(tp), None)
        rays = np.array([[0.2, 0.2, 1, 1e-4, 0, 0, -1, 1e27], [2, 2, 1, 1e-4, 0, 0, -1, 1e27]], np.float32)
        prim, t = np.empty(2, np.int32), np.empty(2, np.float32)
        bary, anyh = np.empty((2, 2), np.float32), np.empty(2, np.int32)
        host_lib.ht_trace(h, oc.fp(rays), 2, oc.fp(prim), oc.fp(t), oc.fp(bary), oc.fp(anyh))
        assert prim[0] == 0 and t[0] == 1.0 and anyh[0] == 1   # ties between coincident copies go to index 0
        assert prim[1] == -1 and anyh[1] == 0
        max_sp = ctypes.c_int()
        assert host_lib.ht_trace4(h, oc.fp(rays), 2, oc.fp(prim), oc.fp(t), oc.fp(bary), oc.fp(anyh), ctypes.byref(max_sp)) == 0
        host_lib.ht_free(h)
        assert prim[0] == 0 and t[0] == 1.0 and anyh[0] == 1
        assert prim[1] == -1 and anyh[1] == 0


def test_host_traversal_far_from_origin(host_lib):
    # the scene shrunk 100x and moved 500 units away from the origin: coordinates on a coarse float
    # grid, so many rays have an exactly zero direction component and start exactly on a box face plane
    data = scenes.single_scene(width=8, height=8, metal_subdiv=3, glass_subdiv=2)
    for m in data.meshes:
        m.positions = np.ascontiguousarray(m.positions * np.float32(0.01) + np.float32(500.0), np.float32)
    tp, _, _ = data.flat_triangles()
    h = host_lib.ht_build(oc.fp(tp), len(tp), None)
    assert h
    rays = edge_and_random_rays(tp, 4000, 5)
    rays[:, 0:3] = rays[:, 0:3] * np.float32(0.01) + np.float32(500.0)
    rays[:, 3] = 1e-6
    d = (tp[np.random.default_rng(5).integers(0, len(tp), len(rays)), 0:3] - rays[:, 0:3]).astype(np.float64)
    rays[:, 4:7] = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    n = len(rays)
    prim4, t4 = np.empty(n, np.int32), np.empty(n, np.float32)
    bary4, anyh4 = np.empty((n, 2), np.float32), np.empty(n, np.int32)
    max_sp = ctypes.c_int()
    assert host_lib.ht_trace4(h, oc.fp(rays), n, oc.fp(prim4), oc.fp(t4), oc.fp(bary4), oc.fp(anyh4), ctypes.byref(max_sp)) == 0
    host_lib.ht_free(h)
    bp, bt, bb, ba = oc.OracleScene(data).trace(rays, brute=True)
    assert np.mean(bp >= 0) > 0.5
    assert np.array_equal(prim4, bp)
    assert np.array_equal(t4.view(np.uint32), bt.view(np.uint32))
    assert np.array_equal(bary4.view(np.uint32), bb.view(np.uint32))
    assert np.array_equal(anyh4, ba)


@pytest.mark.parametrize("plane", [0.0, 0.5, -3.0])
def test_host_traversal_rays_inside_a_box_face_plane(host_lib, plane):
    # triangles with one vertex on the plane x = plane (or y, z) and the rest on one side of it, so that
    # the plane is a face of many boxes; rays with an exactly zero direction component that start on
    # the plane and run inside it, aimed at those vertices: their hits are exactly on box faces
    rng = np.random.default_rng(int(abs(plane) * 10) + 7)
    tris, rays = [], []
    for axis in range(3):
        for k in range(300):
            v0 = rng.uniform(-1, 1, 3).astype(np.float32)
            v0[axis] = plane
            side = -1.0 if k % 2 else 1.0
            v1 = v0 + rng.uniform(0.05, 0.4, 3).astype(np.float32) * side
            v2 = v0 + rng.uniform(0.05, 0.4, 3).astype(np.float32) * side * np.array([1, -1, 1], np.float32)
            v1[axis] = plane + side * rng.uniform(0.05, 0.4)
            v2[axis] = plane + side * rng.uniform(0.05, 0.4)
            tris.append(np.concatenate([v0, v1, v2]))
            o = rng.uniform(-1, 1, 3).astype(np.float32)
            o[axis] = plane
            d = (v0 - o).astype(np.float64)
            d[axis] = 0.0
            d /= np.linalg.norm(d)
            d = d.astype(np.float32)
            d[axis] = 0.0
            rays.append(np.concatenate([o, [1e-5], d, [1e27]]))
    tp = np.ascontiguousarray(np.array(tris, np.float32))
    rays = np.ascontiguousarray(np.array(rays, np.float32))
    h = host_lib.ht_build(oc.fp(tp), len(tp), None)
    n = len(rays)
    prim4, t4 = np.empty(n, np.int32), np.empty(n, np.float32)
    bary4, anyh4 = np.empty((n, 2), np.float32), np.empty(n, np.int32)
    max_sp = ctypes.c_int()
    assert host_lib.ht_trace4(h, oc.fp(rays), n, oc.fp(prim4), oc.fp(t4), oc.fp(bary4), oc.fp(anyh4), ctypes.byref(max_sp)) == 0
    host_lib.ht_free(h)
    # brute force over the same triangles (the oracle's scene needs meshes: one mesh of the triangles)
    from open_rendering_framework_b200 import scene as sc

    P = tp.reshape(-1, 3)
    I = np.arange(len(P), dtype=np.int32).reshape(-1, 3)
    base = scenes.single_scene(width=8, height=8, metal_subdiv=1, glass_subdiv=1)
    data = sc.SceneData(base.integrator, base.camera, base.background, [sc.Mesh(P, I, base.meshes[1].material)], [])
    bp, bt, bb, ba = oc.OracleScene(data).trace(rays, brute=True)
    assert np.mean(bp >= 0) > 0.3
    assert np.array_equal(prim4, bp)
    assert np.array_equal(t4.view(np.uint32), bt.view(np.uint32))
    assert np.array_equal(bary4.view(np.uint32), bb.view(np.uint32))
    assert np.array_equal(anyh4, ba)


def test_host_traversal_over_the_device_builders_tree(host_lib):
    # The device builder's tree (restated by tests/lbvh_host.py) has single-triangle leaves whose boxes end
    # exactly at shared vertices.  Rays aimed at vertices can be reported by the triangle test to hit
    # just outside a triangle (a rounded barycentric), before the box's entry distance when the ray runs
    # nearly parallel to the face it crosses: the box tests' spatial margin keeps those boxes.  Both
    # traversals (stackless BVH2 and 4-wide) must match brute force bit for bit.
    import lbvh_host
    from open_rendering_framework_b200 import scene as sc

    base = scenes.single_scene(width=16, height=16, metal_subdiv=1, glass_subdiv=1)
    meshes = [m for m in base.meshes if not isinstance(m.material, sc.AreaLightMaterial)]
    p, i, nrm, ni = scenes.heightfield(40, extent=1.8, y0=-0.6, seed=4)
    meshes.append(sc.Mesh(p, i, meshes[0].material, nrm, ni))
    data = sc.SceneData(base.integrator, base.camera, base.background, meshes, base.lights)
    tp = np.ascontiguousarray(data.flat_triangles()[0], np.float32)
    nodes, v0, e1, e2 = lbvh_host.build(tp)
    h = host_lib.ht_from_arrays(oc.fp(np.ascontiguousarray(nodes)), len(nodes), oc.fp(v0), oc.fp(e1), oc.fp(e2), len(tp), oc.fp(tp))
    O = oc.OracleScene(data)
    rng = np.random.default_rng(0)
    for seed in range(6):
        # random rays plus rays aimed exactly at triangle vertices and edge midpoints
        rays = edge_and_random_rays(tp, 20000, seed)
        n = len(rays)
        bp, bt, bb, ba = O.trace(rays, brute=True)
        out = [np.empty(n, np.int32), np.empty(n, np.float32), np.empty((n, 2), np.float32), np.empty(n, np.int32)]
        host_lib.ht_trace(h, oc.fp(rays), n, *[oc.fp(a) for a in out])
        out4 = [np.empty(n, np.int32), np.empty(n, np.float32), np.empty((n, 2), np.float32), np.empty(n, np.int32)]
        max_sp = ctypes.c_int()
        assert host_lib.ht_trace4(h, oc.fp(rays), n, *[oc.fp(a) for a in out4], ctypes.byref(max_sp)) == 0
        for p_, t_, b_, a_ in (out, out4):
            assert np.array_equal(p_, bp), (seed, np.flatnonzero(p_ != bp)[:5])
            assert np.array_equal(t_.view(np.uint32), bt.view(np.uint32))
            assert np.array_equal(b_.view(np.uint32), bb.view(np.uint32))
            assert np.array_equal(a_, ba)
    host_lib.ht_free(h)
