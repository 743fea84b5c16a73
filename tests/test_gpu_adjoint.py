"""The adjoint (x2_adjoint, x2.diff.Render) against central finite differences with common random numbers.

Scene: config 4 shrunk (x2_scene_generate 44: a heightfield and icospheres sharing a pool of materials, 16 rect lights
and an environment). Loss = sum over pixels of w * image for fixed random weights w, so dL/dimage = w. Finite
differences re-render the same samples (the same identities, hence the same random numbers) with one parameter moved
by +-h; they see what the adjoint holds fixed (a Russian-roulette or light-choice decision flipping), so the bar is a
few percent on the parameters that matter.
"""
import numpy as np
import pytest

from oracle_lib import x2

pytestmark = pytest.mark.gpu


def _image(scene, spp):
    scene.frame_begin(spp)
    scene.render_frame(0, spp)
    scene.wait()
    scene.audit()
    sums, counts = scene.film()
    return sums[:, :3] / counts[:, None]


@pytest.fixture(scope="module")
def field(ctx):
    s = x2.SyntheticScene(44)
    scene = x2.Scene(ctx, s.desc, s.config)
    d = s.desc
    albedo = np.array([list(d.materials[m].diffuse) for m in range(d.material_count)], np.float64)
    kinds = np.array([d.materials[m].kind for m in range(d.material_count)])
    radiance = np.array([list(d.lights[i].radiance) for i in range(d.light_count)], np.float64)
    return s, scene, albedo, kinds, radiance


def test_adjoint_matches_finite_differences(field):
    import torch

    s, scene, albedo, kinds, radiance = field
    cfg = s.config
    spp = cfg.spp
    pixels = cfg.width * cfg.height
    w = np.random.default_rng(5).random((pixels, 3))
    dev = torch.device("cuda", 0)
    dl = torch.from_numpy(w.astype(np.float32)).to(dev)
    ga = torch.zeros((len(albedo), 3), dtype=torch.float64, device=dev)
    gr = torch.zeros((len(radiance), 3), dtype=torch.float64, device=dev)
    scene.set_params(albedo, radiance)
    torch.cuda.synchronize()
    scene.adjoint(0, spp, dl.data_ptr(), ga.data_ptr(), gr.data_ptr())
    ga, gr = ga.cpu().numpy(), gr.cpu().numpy()
    assert np.all(ga[kinds != x2.MAT_LAMBERT] == 0.0)

    def loss(a, r):
        scene.set_params(a, r)
        return float((_image(scene, spp) * w).sum())

    checked = 0
    lambert = np.flatnonzero(kinds == x2.MAT_LAMBERT)
    for m in lambert[np.argsort(-np.abs(ga[lambert, 0]))][:4]:
        for c in range(3):
            h = 1e-3 * albedo[m, c]
            up, down = albedo.copy(), albedo.copy()
            up[m, c] += h
            down[m, c] -= h
            fd = (loss(up, radiance) - loss(down, radiance)) / (2 * h)
            print(f"albedo[{m},{c}]: adjoint {ga[m, c]:.6g} fd {fd:.6g}")
            assert abs(fd - ga[m, c]) <= 0.03 * abs(ga[m, c]) + 1e-6
            checked += 1
    for i in np.argsort(-np.abs(gr[:, 0]))[:3]:
        h = 1e-3 * radiance[i, 0]
        up, down = radiance.copy(), radiance.copy()
        up[i] += h  # all three channels: the light's colour scaled, d/dh = sum of the channel gradients
        down[i] -= h
        fd = (loss(albedo, up) - loss(albedo, down)) / (2 * h)
        want = gr[i].sum()
        print(f"radiance[{i}]: adjoint {want:.6g} fd {fd:.6g}")
        assert abs(fd - want) <= 0.03 * abs(want) + 1e-6
        checked += 1
    scene.set_params(albedo, radiance)
    assert checked == 15


def test_autograd_function(field):
    import torch
    from x2.diff import render

    s, scene, albedo, kinds, radiance = field
    dev = torch.device("cuda", 0)
    a = torch.tensor(albedo, dtype=torch.float32, device=dev, requires_grad=True)
    r = torch.tensor(radiance, dtype=torch.float32, device=dev, requires_grad=True)
    spp = s.config.spp
    target = render(scene, a.detach() * 0.5, r.detach(), 0, spp).detach()
    image = render(scene, a, r, 0, spp)
    loss = ((image - target) ** 2).sum()
    loss.backward()
    assert a.grad is not None and r.grad is not None
    assert torch.isfinite(a.grad).all() and torch.isfinite(r.grad).all()
    # Halving the albedos darkened the target: the loss falls as the Lambert albedos fall.
    lam = torch.tensor(kinds == x2.MAT_LAMBERT, device=dev)
    assert (a.grad[lam].sum() > 0).item()
    scene.set_params(albedo, radiance)
