"""Adjoint (path replay backprop) gradients on the GPU against FP64 references.

The differentiated estimator keeps the forward render's sampling fixed (pt_render_adjoint).  Its
FP64 reference is the oracle's path tapes: the same camera paths traced by the CPU restatement, with
what every vertex adds and multiplies recorded, re-evaluated in FP64 (orc_tape_eval) -- once
analytically (path replay on the stored vertices) and once by central finite differences (h = 1e-4)
of the loss itself.  The tape's analytic gradient is pinned to its finite differences on the CPU
(tests/test_oracle_pin.py); here the GPU's FP32 gradient is compared with both.  Bars: at least 95%
of 64 random parameters within 1e-3 relative of the FD gradient (all six sigmas among them), and the
gradient vectors within 1e-3 relative in the L2 sense.
"""
import numpy as np
import pytest

from oracle import oracle_ctypes as oc
from open_rendering_framework_b200 import scenes

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_adjoint_matches_fp64_finite_differences():
    from open_rendering_framework_b200 import diff

    W = H = 32
    spp = 4
    data, (dif, met, tr) = scenes.inverse_scene(W, H, subdiv=3, tex_res=30, probe_samples=64, seed=3)
    DS = diff.DiffScene(data, dif, met, tr)
    albedo = torch.from_numpy(dif.texture.copy()).cuda().requires_grad_()
    rough = torch.from_numpy(met.texture.copy()).cuda().requires_grad_()
    sig = np.r_[np.asarray(tr.absorption, np.float32), np.asarray(tr.scattering, np.float32)]
    sigma = torch.from_numpy(sig.copy()).cuda().requires_grad_()
    img = diff.render(DS, spp, albedo, rough, sigma)
    target = (img.detach() * 0.6 + 0.02).contiguous()
    loss = ((img - target) ** 2).sum()
    loss.backward()
    g_gpu = np.concatenate([albedo.grad.cpu().numpy().ravel(), rough.grad.cpu().numpy().ravel(), sigma.grad.cpu().numpy()]).astype(np.float64)
    st = DS.stats()
    assert st.gather_overflows == 0

    # FP64 references from the oracle's tapes of the same paths
    O = oc.OracleScene(data)
    O.record(True)
    acc, _ = O.render(0, spp, accum=np.zeros((H, W, 4), np.float32), threads=8)
    tex_off, mat_off, n = O.param_layout([dif, met, tr])
    P = np.concatenate([dif.texture.ravel(), met.texture.ravel(), sig]).astype(np.float64)
    tgt = target.cpu().numpy().reshape(-1, 3).astype(np.float64)
    img_gpu = img.detach().cpu().numpy().reshape(-1, 3).astype(np.float64)
    img64, g64 = O.tape_eval(P, tex_off, mat_off, dimg=2.0 * (img_gpu - tgt))
    assert np.max(np.abs(img64 - img_gpu) / np.maximum(np.abs(img_gpu), 1e-3)) < 2e-3
    # whole gradient against the FP64 analytic one (same image gradient)
    l2 = np.linalg.norm(g_gpu - g64) / np.linalg.norm(g64)
    print("GPU vs FP64 analytic gradient: relative L2", l2, "of", n, "parameters")
    assert l2 < 1e-3

    def loss64(Pv):
        im, _ = O.tape_eval(Pv, tex_off, mat_off)
        return np.sum((im - tgt) ** 2)

    rng = np.random.default_rng(7)
    nz = np.nonzero(np.abs(g64) > 1e-6 * np.max(np.abs(g64)))[0]
    pick = list(rng.choice(nz[nz < n - 6], 58, replace=False)) + list(range(n - 6, n))
    h = 1e-4
    rel = []
    for i in pick:
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += h
        Pm[i] -= h
        fd = (loss64(Pp) - loss64(Pm)) / (2.0 * h)
        rel.append(abs(g_gpu[i] - fd) / max(abs(fd), 1e-12))
    rel = np.array(rel)
    print("GPU vs FP64 central FD on 64 parameters: within 1e-3:", np.mean(rel <= 1e-3), "max", rel.max(), "sigma", rel[-6:])
    assert np.mean(rel <= 1e-3) >= 0.95
    assert np.all(rel[-6:] <= 1e-3)
    DS.close()


def test_adjoint_same_under_both_schedules():
    """The overlapped schedule (shading classes and shadow rays on streams of their own) and the
    in-order one give the same image and the same gradients: each path's replay is its own; only the
    order of the gradient atomics differs, so the gradients agree to float-summation order."""
    from open_rendering_framework_b200 import diff

    data, (dif, met, tr) = scenes.inverse_scene(24, 24, subdiv=3, tex_res=16, probe_samples=32, seed=5)
    out = []
    for overlap in (1, 0):
        DS = diff.DiffScene(data, dif, met, tr)
        DS.R.set_option("overlap", overlap)
        albedo = torch.from_numpy(dif.texture.copy()).cuda().requires_grad_()
        rough = torch.from_numpy(met.texture.copy()).cuda().requires_grad_()
        sig = np.r_[np.asarray(tr.absorption, np.float32), np.asarray(tr.scattering, np.float32)]
        sigma = torch.from_numpy(sig.copy()).cuda().requires_grad_()
        img = diff.render(DS, 3, albedo, rough, sigma)
        (img ** 2).sum().backward()
        out.append((img.detach().cpu().numpy(), albedo.grad.cpu().numpy(), rough.grad.cpu().numpy(), sigma.grad.cpu().numpy()))
        DS.close()
    assert np.array_equal(out[0][0].view(np.uint32), out[1][0].view(np.uint32))
    for a, b in zip(out[0][1:], out[1][1:]):
        assert np.allclose(a, b, rtol=1e-4, atol=1e-6 * np.max(np.abs(b))), np.max(np.abs(a - b))


def test_adjoint_requires_differentiable_forward():
    from open_rendering_framework_b200 import _native as nat
    from open_rendering_framework_b200 import scene as sc

    data, _ = scenes.inverse_scene(16, 16, subdiv=1, tex_res=12, probe_samples=16)
    R = sc.Renderer(data)
    R.render(1)
    d = torch.zeros((16, 16, 4), dtype=torch.float32, device="cuda")
    with pytest.raises(nat.PtError):
        nat.call("pt_render_adjoint", R.ctx, 0, 1, d.data_ptr())
    nat.call("pt_set_option", R.ctx, b"differentiable", 1)
    nat.call("pt_render_frames", R.ctx, 0, 2)
    with pytest.raises(nat.PtError):
        nat.call("pt_render_adjoint", R.ctx, 0, 3, d.data_ptr())  # not the frames rendered
    nat.call("pt_render_adjoint", R.ctx, 0, 2, d.data_ptr())
    R.sync()
    R.close()
