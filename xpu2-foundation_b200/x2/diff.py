"""Differentiable rendering behind torch.autograd (config 4): the image of a frame as a function of each material's
albedo and roughness and each light's radiance.

Forward renders the frame with the parameters set (x2_scene_set_params, then the wavefront form) and returns the
film's mean image; backward calls the adjoint (x2_adjoint), which replays each sample's path from its identity and
credits each contribution to the light it reached and the Lambert and GGX vertices it passed. The adjoint takes its own
samples (`adjoint_first`, `adjoint_count`), decorrelated from the primal's unless the caller picks the same ones.
"""
import numpy as np
import torch


def _host(t):
    return None if t is None else t.detach().double().cpu().numpy()


class Render(torch.autograd.Function):
    @staticmethod
    def forward(ctx, albedo, radiance, roughness, scene, first, count, adjoint_first, adjoint_count):
        scene.set_params(_host(albedo), _host(radiance), _host(roughness))
        scene.frame_begin(count)
        scene.render_frame_wavefront(first, count)
        scene.wait()
        sums, counts = scene.film()
        cfg = scene.config
        image = (sums[:, :3] / np.maximum(counts, 1)[:, None]).reshape(cfg.height, cfg.width, 3)
        ctx.scene = scene
        ctx.adjoint = (adjoint_first, adjoint_count)
        ctx.params = [(p.shape, p.dtype, p.device) if p is not None else None for p in (albedo, radiance, roughness)]
        return torch.from_numpy(image.astype(np.float32)).to(albedo.device)

    @staticmethod
    def backward(ctx, grad_image):
        dev = torch.device("cuda", torch.cuda.current_device())
        dl = grad_image.detach().to(dev, torch.float32).contiguous()
        (a_shape, _, _), (r_shape, _, _) = ctx.params[0], ctx.params[1]
        ga = torch.zeros(a_shape, dtype=torch.float64, device=dev)
        gr = torch.zeros(r_shape, dtype=torch.float64, device=dev)
        gg = torch.zeros(ctx.params[2][0], dtype=torch.float64, device=dev) if ctx.params[2] is not None else None
        first, count = ctx.adjoint
        torch.cuda.synchronize()
        ctx.scene.adjoint(first, count, dl.data_ptr(), ga.data_ptr(), gr.data_ptr(), gg.data_ptr() if gg is not None else None)
        out = []
        for g, p in zip((ga, gr, gg), ctx.params):
            out.append(None if p is None else g.to(p[2], p[1]))
        return (*out, None, None, None, None, None)


def render(scene, albedo, radiance, first, count, adjoint_first=None, adjoint_count=None, roughness=None):
    """The frame's image (height x width x 3, float32) as a differentiable function of albedo (materials x 3), radiance
    (lights x 3) and, when given, roughness (materials). The adjoint uses samples [adjoint_first, adjoint_first +
    adjoint_count) (default: the primal's own)."""
    return Render.apply(albedo, radiance, roughness, scene, first, count, first if adjoint_first is None else adjoint_first,
                        count if adjoint_count is None else adjoint_count)
