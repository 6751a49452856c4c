"""Batched rendering (pt_batch_*): several scenes in one wavefront pass, replayed from a CUDA graph.

A batched render of frames [f, f+n) of a scene must leave exactly the image pt_render_frames(ctx, f,
n) leaves -- the same kernels on the same seeds, only the path-id layout differs -- so every check
here is bit-exact against the scenes rendered one by one (those with every launch in order on one
stream, the batch with its shading classes and shadow rays overlapped on two more streams, inside the
captured graph too).
"""
import numpy as np
import pytest

from open_rendering_framework_b200 import scene as sc
from open_rendering_framework_b200 import scenes

pytestmark = pytest.mark.gpu


def small_batch(n=6, seed=5):
    out = [scenes.batch_scene(k, seed, size_scale=1 / 16, spp_scale=0.08, probe_samples=64) for k in range(n)]
    # make sure every material kind is present
    kinds = {info["material"] for _, _, info in out}
    k = n
    while kinds != set(scenes.BATCH_MATERIALS):
        d, spp, info = scenes.batch_scene(k, seed, size_scale=1 / 16, spp_scale=0.08, probe_samples=64)
        if info["material"] not in kinds:
            out.append((d, spp, info))
            kinds.add(info["material"])
        k += 1
    return out


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.mark.parametrize("use_graph", [1, 0])
def test_batched_render_equals_scene_by_scene(use_graph):
    S = small_batch()
    solo = []
    for data, spp, _ in S:
        R = sc.Renderer(data)
        R.set_option("overlap", 0)  # the in-order schedule; the batch engine overlaps (the default)
        R.render(spp)
        R.render(spp)
        solo.append(R.readback())
        R.close()
    Rs = [sc.Renderer(data) for data, _, _ in S]
    B = sc.Batch(Rs, [spp for _, spp, _ in S])
    B.set_option("use_graph", use_graph)
    B.render()
    B.render()  # second render: replays the captured graph with the next frames
    st = B.stats()
    assert st.path_samples == sum(d.camera.width * d.camera.height * spp for d, spp, _ in S)
    for R, ref, (_, spp, info) in zip(Rs, solo, S):
        assert R.frame == 2 * spp
        got = R.readback()
        assert np.array_equal(bits(got), bits(ref)), info
    B.close()
    for R in Rs:
        R.close()


def test_graph_replay_follows_changed_scenes():
    """A scene changed between two batched renders (here its integrator's scene epsilon, which the
    traversal kernels of a one-scene chunk receive by value) makes the batch capture its graph again, so
    the second render equals scene-by-scene renders that made the same change."""
    S = small_batch(3, seed=11)
    eps2 = 3e-3
    eps1 = [data.integrator.scene_epsilon for data, _, _ in S]

    def run(batched):
        for (data, _, _), e in zip(S, eps1):
            data.integrator.scene_epsilon = e
        Rs = [sc.Renderer(data) for data, _, _ in S]
        B = sc.Batch(Rs, [spp for _, spp, _ in S]) if batched else None
        if B:
            B.set_option("max_paths_in_flight", 64)  # every chunk one frame of one scene
        for step in range(2):
            if step == 1:
                for R in Rs:
                    R.data.integrator.scene_epsilon = eps2
                    R.apply_integrator()
            if batched:
                B.render()
            else:
                for R, (_, spp, _) in zip(Rs, S):
                    R.render(spp)
        imgs = [R.readback() for R in Rs]
        if B:
            B.close()
        for R in Rs:
            R.close()
        return imgs

    for a, b, (_, _, info) in zip(run(True), run(False), S):
        assert np.array_equal(bits(a), bits(b)), info


def test_sequential_mode_and_autotune():
    S = small_batch(4, seed=9)
    Rs = [sc.Renderer(data) for data, _, _ in S]
    B = sc.Batch(Rs, [spp for _, spp, _ in S])
    res = B.autotune(frames_per_trial=1)
    assert res.trials >= 5 and res.refill in (16, 20, 24) and res.best_mpaths_per_s > 0
    assert all(R.frame == 0 for R in Rs)
    B.render()
    batched = [R.readback() for R in Rs]
    Rs2 = [sc.Renderer(data) for data, _, _ in S]
    B2 = sc.Batch(Rs2, [spp for _, spp, _ in S])
    B2.render_sequential()
    for a, R in zip(batched, Rs2):
        assert np.array_equal(bits(a), bits(R.readback()))
    B.close()
    B2.close()
    for R in Rs + Rs2:
        R.close()


def test_batch_rejects_bad_scenes():
    import ctypes

    from open_rendering_framework_b200 import _native as nat

    data, spp, _ = scenes.batch_scene(0, 1, size_scale=1 / 16, spp_scale=0.1)
    R = sc.Renderer(data)
    B = sc.Batch([R], [spp])
    with pytest.raises(nat.PtError):
        nat.call("pt_batch_add", B.b, R.ctx, 1)  # already in the batch
    with pytest.raises(nat.PtError):
        nat.call("pt_batch_add", B.b, R.ctx, 0)
    empty = ctypes.c_void_p()
    nat.call("pt_batch_create", 0, ctypes.byref(empty))
    with pytest.raises(nat.PtError):
        nat.call("pt_batch_render", empty)
    nat.call("pt_batch_destroy", empty)
    B.close()
    R.close()


def test_profiled_batch_pass_times_extend_and_gather_and_keeps_images():
    # option "profile": events around every extend and gather launch of a pass without the graph; the
    # pass (in-order schedule) leaves the same images as the graph replay of the same frames
    S = small_batch()
    spp = [p for _, p, _ in S]
    images = []
    for profile in (0, 1):
        Rs = [sc.Renderer(data) for data, _, _ in S]
        B = sc.Batch(Rs, spp)
        if profile:
            B.set_option("use_graph", 0)
            B.set_option("profile", 1)
        B.render()
        st = B.stats()
        if profile:
            assert st.extend_ms > 0.0 and st.gather_ms > 0.0 and st.dipole_pairs > 0
            assert st.extend_ms + st.gather_ms <= st.gpu_ms * 1.001
        images.append([R.readback() for R in Rs])
        B.close()
        for R in Rs:
            R.close()
    for a, b in zip(*images):
        assert np.array_equal(bits(a), bits(b))
