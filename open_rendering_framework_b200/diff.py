"""Differentiable rendering through the C ABI, wrapped as a torch.autograd.Function.

The forward pass is pt_render_frames with the "differentiable" option (each camera path keeps its
radiance and its dipole-gather values); the backward pass is pt_render_adjoint (path replay
backprop: the same paths replayed with the same random numbers, sampling detached).  Parameters are
torch CUDA tensors bound to the scene without copies: the albedo texture of a diffuse material
[H, W, 3], the roughness texture of a GGX conductor [H, W], and (sigma_a RGB, sigma_s' RGB) of a
translucent material (standard dipole) in the units of TranslucentMaterial.

The adjoint uses the state of the most recent differentiable forward render of the same scene, so
call backward before rendering that scene again.
"""
import ctypes

import torch

from . import _native as nat
from . import scene as sc


class DiffScene:
    """A Renderer with bound parameter tensors (see the module docstring)."""

    def __init__(self, data, albedo_material, roughness_material, translucent_material, device=0):
        self.R = sc.Renderer(data, device=device)
        nat.call("pt_set_option", self.R.ctx, b"differentiable", 1)
        self.device = device
        self.tex_albedo = self.R.texture_ids[id(albedo_material)]
        self.tex_rough = self.R.texture_ids[id(roughness_material)]
        self.trans = translucent_material
        self.mid_trans = self.R.material_ids[id(translucent_material)]
        self.W, self.H = data.camera.width, data.camera.height
        self._bound = None

    def bind(self, albedo, rough, sigma):
        """Points the textures at the tensors' memory and sets the translucent material's sigmas."""
        assert albedo.is_cuda and albedo.dtype == torch.float32 and albedo.is_contiguous()
        assert rough.is_cuda and rough.dtype == torch.float32 and rough.is_contiguous()
        torch.cuda.synchronize(self.device)
        nat.call("pt_texture_bind", self.R.ctx, self.tex_albedo, albedo.data_ptr())
        nat.call("pt_texture_bind", self.R.ctx, self.tex_rough, rough.data_ptr())
        s = [float(x) for x in sigma.detach().double().cpu()]
        g = self.trans.meancosine
        self.trans.absorption = tuple(s[:3])
        self.trans.scattering = tuple(s[3 + c] / (1.0 - g[c]) for c in range(3))
        self.R.update_material(self.trans)
        self._bound = (albedo, rough)

    def render(self, spp):
        """Frames 0 .. spp-1 into the running mean; returns the image [H, W, 3]."""
        nat.call("pt_render_frames", self.R.ctx, 0, int(spp))
        self.R.frame = int(spp)
        out = torch.empty((self.H, self.W, 4), dtype=torch.float32, device="cuda:%d" % self.device)
        nat.call("pt_readback_device", self.R.ctx, out.data_ptr())
        self.R.sync()
        return out[..., :3].contiguous()

    def adjoint(self, spp, grad_image):
        """Gradients (albedo [H,W,3], roughness [H,W], sigma [6]) of a loss whose gradient with
        respect to the image is grad_image [H, W, 3]."""
        albedo, rough = self._bound
        dev = albedo.device
        dimg = torch.zeros((self.H, self.W, 4), dtype=torch.float32, device=dev)
        dimg[..., :3] = grad_image.to(torch.float32)
        ga = torch.zeros_like(albedo)
        gr = torch.zeros_like(rough)
        gs = torch.zeros(6, dtype=torch.float32, device=dev)
        torch.cuda.synchronize(self.device)
        nat.call("pt_texture_bind_grad", self.R.ctx, self.tex_albedo, ga.data_ptr())
        nat.call("pt_texture_bind_grad", self.R.ctx, self.tex_rough, gr.data_ptr())
        nat.call("pt_material_bind_sigma_grad", self.R.ctx, self.mid_trans, gs.data_ptr())
        nat.call("pt_render_adjoint", self.R.ctx, 0, int(spp), dimg.data_ptr())
        self.R.sync()
        nat.call("pt_texture_bind_grad", self.R.ctx, self.tex_albedo, None)
        nat.call("pt_texture_bind_grad", self.R.ctx, self.tex_rough, None)
        nat.call("pt_material_bind_sigma_grad", self.R.ctx, self.mid_trans, None)
        return ga, gr, gs

    def stats(self):
        return self.R.stats()

    def close(self):
        self.R.close()


class RenderFunction(torch.autograd.Function):
    """image = RenderFunction.apply(scene, spp, albedo, roughness, sigma)."""

    @staticmethod
    def forward(ctx, scene, spp, albedo, rough, sigma):
        scene.bind(albedo, rough, sigma)
        img = scene.render(spp)
        ctx.scene, ctx.spp = scene, spp
        ctx.save_for_backward(albedo, rough, sigma)
        return img

    @staticmethod
    def backward(ctx, grad_img):
        albedo, rough, sigma = ctx.saved_tensors
        ga, gr, gs = ctx.scene.adjoint(ctx.spp, grad_img.contiguous())
        return None, None, ga, gr, gs.to(sigma.dtype)


def render(scene, spp, albedo, rough, sigma):
    return RenderFunction.apply(scene, spp, albedo, rough, sigma)
