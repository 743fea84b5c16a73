"""Differentiable rendering behind torch.autograd (config 4): the image of a frame as a function of each material's
albedo and each light's radiance.

Forward renders the frame with the parameters set (x2_scene_set_params, then the wavefront form) and returns the
film's mean image; backward calls the adjoint (x2_adjoint), which replays each sample's path from its identity and
credits each contribution to the light it reached and the Lambert vertices it passed. The adjoint takes its own
samples (`adjoint_first`, `adjoint_count`), decorrelated from the primal's unless the caller picks the same ones.
"""
import numpy as np
import torch


class Render(torch.autograd.Function):
    @staticmethod
    def forward(ctx, albedo, radiance, scene, first, count, adjoint_first, adjoint_count):
        scene.set_params(albedo.detach().double().cpu().numpy(), radiance.detach().double().cpu().numpy())
        scene.frame_begin(count)
        scene.render_frame_wavefront(first, count)
        scene.wait()
        sums, counts = scene.film()
        cfg = scene.config
        image = (sums[:, :3] / np.maximum(counts, 1)[:, None]).reshape(cfg.height, cfg.width, 3)
        ctx.scene = scene
        ctx.adjoint = (adjoint_first, adjoint_count)
        ctx.shapes = (albedo.shape, radiance.shape, albedo.dtype, radiance.dtype, albedo.device)
        return torch.from_numpy(image.astype(np.float32)).to(albedo.device)

    @staticmethod
    def backward(ctx, grad_image):
        a_shape, r_shape, a_dtype, r_dtype, device = ctx.shapes
        dev = torch.device("cuda", torch.cuda.current_device())
        dl = grad_image.detach().to(dev, torch.float32).contiguous()
        ga = torch.zeros(a_shape, dtype=torch.float64, device=dev)
        gr = torch.zeros(r_shape, dtype=torch.float64, device=dev)
        first, count = ctx.adjoint
        torch.cuda.synchronize()
        ctx.scene.adjoint(first, count, dl.data_ptr(), ga.data_ptr(), gr.data_ptr())
        return ga.to(device, a_dtype), gr.to(device, r_dtype), None, None, None, None, None


def render(scene, albedo, radiance, first, count, adjoint_first=None, adjoint_count=None):
    """The frame's image (height x width x 3, float32) as a differentiable function of albedo (materials x 3) and
    radiance (lights x 3). The adjoint uses samples [adjoint_first, adjoint_first + adjoint_count) (default: the
    primal's own)."""
    return Render.apply(albedo, radiance, scene, first, count, first if adjoint_first is None else adjoint_first,
                        count if adjoint_count is None else adjoint_count)
