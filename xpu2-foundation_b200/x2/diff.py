"""Differentiable rendering behind torch.autograd (config 4): the image of a frame as a function of each material's
albedo and roughness, each light's radiance and the texels of the scene's first texture.

Forward renders the frame with the parameters set (x2_scene_set_params, x2_scene_set_texture, then the wavefront form)
and returns the film's mean image; backward calls the adjoint (x2_adjoint), which replays each sample's path from its
identity and credits each contribution to the light it reached, the Lambert vertices (and the texels their lookups
read) and the GGX vertices it passed. The adjoint takes its own samples (`adjoint_first`, `adjoint_count`),
decorrelated from the primal's unless the caller picks the same ones.
"""
import numpy as np
import torch


def _host(t):
    return None if t is None else t.detach().double().cpu().numpy()


class Render(torch.autograd.Function):
    @staticmethod
    def forward(ctx, albedo, radiance, roughness, texture, scene, first, count, adjoint_first, adjoint_count):
        scene.set_params(_host(albedo), _host(radiance), _host(roughness))
        if texture is not None:
            scene.set_texture(0, _host(texture))
        scene.frame_begin(count)
        scene.render_frame_wavefront(first, count)
        scene.wait()
        sums, counts = scene.film()
        cfg = scene.config
        image = (sums[:, :3] / np.maximum(counts, 1)[:, None]).reshape(cfg.height, cfg.width, 3)
        ctx.scene = scene
        ctx.adjoint = (adjoint_first, adjoint_count)
        ctx.params = [(p.shape, p.dtype, p.device) if p is not None else None for p in (albedo, radiance, roughness, texture)]
        return torch.from_numpy(image.astype(np.float32)).to(albedo.device)

    @staticmethod
    def backward(ctx, grad_image):
        dev = torch.device("cuda", torch.cuda.current_device())
        dl = grad_image.detach().to(dev, torch.float32).contiguous()
        grads = [torch.zeros(p[0], dtype=torch.float64, device=dev) if p is not None else None for p in ctx.params]
        ga, gr, gg, gt = grads
        first, count = ctx.adjoint
        torch.cuda.synchronize()
        ctx.scene.adjoint(first, count, dl.data_ptr(), ga.data_ptr(), gr.data_ptr(), gg.data_ptr() if gg is not None else None,
                          d_texture_grad=gt.data_ptr() if gt is not None else None)
        out = [None if p is None else g.to(p[2], p[1]) for g, p in zip(grads, ctx.params)]
        return (*out, None, None, None, None, None)


def render(scene, albedo, radiance, first, count, adjoint_first=None, adjoint_count=None, roughness=None, texture=None):
    """The frame's image (height x width x 3, float32) as a differentiable function of albedo (materials x 3), radiance
    (lights x 3) and, when given, roughness (materials) and the scene's first texture (height x width x 3; its
    gradient covers the first texture's texels only when the scene has one texture). The adjoint uses samples
    [adjoint_first, adjoint_first + adjoint_count) (default: the primal's own)."""
    return Render.apply(albedo, radiance, roughness, texture, scene, first, count, first if adjoint_first is None else adjoint_first,
                        count if adjoint_count is None else adjoint_count)
