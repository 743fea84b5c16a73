"""The adjoint (x2_adjoint, x2.diff.Render) against central finite differences with common random numbers.

Scene: config 4 shrunk (x2_scene_generate 44: a heightfield and icospheres sharing a pool of materials, 16 rect lights
and an environment). Loss = sum over pixels of w * image for fixed random weights w, so dL/dimage = w. Finite
differences re-render the same samples (the same identities, hence the same random numbers) with one parameter moved
by +-h; they see what the adjoint holds fixed (a Russian-roulette or light-choice decision flipping, whose effect on
the differences grows as 1 / h): both estimate the same derivative with their own noise, so the check takes 256
samples a pixel, a 5% step and a bar of 3% of the gradient plus 0.2% of the largest of its kind. For roughness the finite differences also move the GGX samples'
directions (the adjoint holds them fixed), and a direction that crosses an edge moves the image by a step: both
estimate the same derivative but the differences are noisy, so that check takes many samples, a wider step and the
moderately rough materials (near-mirror lobes make both estimates noisy), with a 10% bar. The exact check of the
adjoint's arithmetic is the one against the FP64 CPU adjoint of the same samples (last test).
"""
import numpy as np
import pytest

from oracle_lib import x2

pytestmark = pytest.mark.gpu


def _image(scene, spp):
    scene.frame_begin(spp)
    scene.render_frame(0, spp)
    scene.wait()
    sums, counts = scene.film()
    scene.audit(np.full(len(counts), spp, np.uint32))
    return sums[:, :3] / counts[:, None]


@pytest.fixture(scope="module")
def field(ctx):
    s = x2.SyntheticScene(44)
    scene = x2.Scene(ctx, s.desc, s.config)
    d = s.desc
    albedo = np.array([list(d.materials[m].diffuse) for m in range(d.material_count)], np.float64)
    kinds = np.array([d.materials[m].kind for m in range(d.material_count)])
    radiance = np.array([list(d.lights[i].radiance) for i in range(d.light_count)], np.float64)
    roughness = np.array([d.materials[m].roughness for m in range(d.material_count)], np.float64)
    return s, scene, albedo, kinds, radiance, roughness


def test_adjoint_matches_finite_differences(field):
    import torch

    s, scene, albedo, kinds, radiance, _ = field
    cfg = s.config
    spp = 256
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
            h = 5e-2 * albedo[m, c]
            up, down = albedo.copy(), albedo.copy()
            up[m, c] += h
            down[m, c] -= h
            fd = (loss(up, radiance) - loss(down, radiance)) / (2 * h)
            print(f"albedo[{m},{c}]: adjoint {ga[m, c]:.6g} fd {fd:.6g}")
            assert abs(fd - ga[m, c]) <= 0.03 * abs(ga[m, c]) + 2e-3 * np.abs(ga[lambert]).max()
            checked += 1
    for i in np.argsort(-np.abs(gr[:, 0]))[:3]:
        h = 5e-2 * radiance[i, 0]
        up, down = radiance.copy(), radiance.copy()
        up[i] += h  # all three channels: the light's colour scaled, d/dh = sum of the channel gradients
        down[i] -= h
        fd = (loss(albedo, up) - loss(albedo, down)) / (2 * h)
        want = gr[i].sum()
        print(f"radiance[{i}]: adjoint {want:.6g} fd {fd:.6g}")
        assert abs(fd - want) <= 0.03 * abs(want) + 2e-3 * np.abs(gr.sum(1)).max()
        checked += 1
    scene.set_params(albedo, radiance)
    assert checked == 15


def test_roughness_matches_finite_differences(field):
    import torch

    s, scene, albedo, kinds, radiance, roughness = field
    cfg = s.config
    spp = 1024
    pixels = cfg.width * cfg.height
    w = np.random.default_rng(6).random((pixels, 3))
    dev = torch.device("cuda", 0)
    dl = torch.from_numpy(w.astype(np.float32)).to(dev)
    ga = torch.zeros((len(albedo), 3), dtype=torch.float64, device=dev)
    gr = torch.zeros((len(radiance), 3), dtype=torch.float64, device=dev)
    gg = torch.zeros(len(roughness), dtype=torch.float64, device=dev)
    scene.set_params(albedo, radiance, roughness)
    torch.cuda.synchronize()
    scene.adjoint(0, spp, dl.data_ptr(), ga.data_ptr(), gr.data_ptr(), gg.data_ptr())
    gg = gg.cpu().numpy()
    assert np.all(gg[kinds != x2.MAT_GGX] == 0.0)
    ggx = np.flatnonzero((kinds == x2.MAT_GGX) & (roughness ** 2 > 0.001))
    assert len(ggx) > 0 and np.any(gg[ggx] != 0.0)
    rough = ggx[(roughness[ggx] >= 0.2) & (roughness[ggx] <= 0.9)]
    assert len(rough) >= 3

    def loss(g):
        scene.set_params(roughness=g)
        return float((_image(scene, spp) * w).sum())

    for m in rough[np.argsort(-np.abs(gg[rough]))][:3]:
        h = 1e-2
        up, down = roughness.copy(), roughness.copy()
        up[m] += h
        down[m] -= h
        fd = (loss(up) - loss(down)) / (2 * h)
        print(f"roughness[{m}] = {roughness[m]:.3f}: adjoint {gg[m]:.6g} fd {fd:.6g}")
        # The differences' noise is absolute (edge crossings): 10% of the gradient or 1% of the largest one.
        assert abs(fd - gg[m]) <= 0.1 * abs(gg[m]) + 0.01 * np.abs(gg[rough]).max()
    scene.set_params(roughness=roughness)


def test_autograd_function(field):
    import torch
    from x2.diff import render

    s, scene, albedo, kinds, radiance, roughness = field
    dev = torch.device("cuda", 0)
    a = torch.tensor(albedo, dtype=torch.float32, device=dev, requires_grad=True)
    r = torch.tensor(radiance, dtype=torch.float32, device=dev, requires_grad=True)
    g = torch.tensor(roughness, dtype=torch.float32, device=dev, requires_grad=True)
    tex0 = s.texture(0)
    t = torch.tensor(tex0, dtype=torch.float32, device=dev, requires_grad=True)
    spp = s.config.spp
    target = render(scene, a.detach() * 0.5, r.detach(), 0, spp, roughness=g.detach(), texture=t.detach() * 0.5).detach()
    image = render(scene, a, r, 0, spp, roughness=g, texture=t)
    loss = ((image - target) ** 2).sum()
    loss.backward()
    assert a.grad is not None and r.grad is not None and g.grad is not None and t.grad is not None
    assert t.grad.shape == t.shape
    for grad in (a.grad, r.grad, g.grad, t.grad):
        assert torch.isfinite(grad).all()
    assert (g.grad[torch.tensor(kinds != x2.MAT_GGX, device=dev)] == 0).all()
    # The target's texture is halved too: the loss falls as the texels fall.
    assert (t.grad.sum() > 0).item()
    scene.set_texture(0, tex0)
    # Halving the albedos darkened the target: the loss falls as the Lambert albedos fall.
    lam = torch.tensor(kinds == x2.MAT_LAMBERT, device=dev)
    assert (a.grad[lam].sum() > 0).item()
    scene.set_params(albedo, radiance, roughness)


def test_adjoint_matches_fp64_cpu_adjoint(field):
    """The device adjoint (FP32 arithmetic, FP32 atomics into per-block partials, FP64 reduction) against the FP64 CPU
    adjoint of the same samples (oracle/adjoint64.h: the estimator restated in double, the reference's sampler): 64
    seeded random parameters among the Lambert albedo channels, GGX roughnesses and light radiance channels.

    A gradient is a sum of credits; its mass is the sum of the credits' magnitudes. Two things separate the device's
    sum from the FP64 one in proportion to the mass, not to the sum: the primal's float rounding (about 1e-3 of a
    credit for a glossy lobe's value, which the primal computes in float as the reference does, against the exact
    one), and the rare sample that takes another roulette or visibility decision in double than in float (its path's
    credits then differ; their share falls as 1/sqrt(samples)). So over 1,048,576 samples each parameter must be within
    1% of its FP64 value plus 1e-3 of its mass, and each kind's gradients of conditioning (mass over value) up to 10
    within 1% in L2. Near-mirror GGX
    roughnesses are near-cancelling sums (credits of hundreds either way from dlog D) whose mass is up to hundreds of
    times their value: the mass term is what holds them."""
    import oracle_lib
    import torch

    s, scene, albedo, kinds, radiance, roughness = field
    if not oracle_lib.have_reference():
        pytest.skip("oracle/_ref not built")
    cfg = s.config
    spp = 256
    pixels = cfg.width * cfg.height
    w = np.random.default_rng(7).random((pixels, 3)).astype(np.float32)
    dev = torch.device("cuda", 0)
    dl = torch.from_numpy(w).to(dev)
    ga = torch.zeros((len(albedo), 3), dtype=torch.float64, device=dev)
    gr = torch.zeros((len(radiance), 3), dtype=torch.float64, device=dev)
    gg = torch.zeros(len(roughness), dtype=torch.float64, device=dev)
    scene.set_params(albedo, radiance, roughness)
    scene.set_texture(0, s.texture(0))
    torch.cuda.synchronize()
    scene.adjoint(0, spp, dl.data_ptr(), ga.data_ptr(), gr.data_ptr(), gg.data_ptr())
    ga, gr, gg = ga.cpu().numpy(), gr.cpu().numpy(), gg.cpu().numpy()
    ref = oracle_lib.Reference(s)
    ca, cg, cr, _, (ma, mg, mr) = oracle_lib.adjoint64(ref, 0, spp, w, params=(albedo, roughness, radiance), masses=True)
    ref.close()
    lam = np.flatnonzero(kinds == x2.MAT_LAMBERT)
    ggx = np.flatnonzero(kinds == x2.MAT_GGX)
    for m in ggx:
        print(f"roughness[{m}] r={roughness[m]:.3f} device {gg[m]:.6g} fp64 {cg[m]:.6g} mass {mg[m]:.4g}")
    cands = [("albedo", (m, c)) for m in lam for c in range(3)] + [("roughness", (m,)) for m in ggx] + \
            [("radiance", (i, c)) for i in range(len(radiance)) for c in range(3)]
    dev_g = {"albedo": ga, "roughness": gg, "radiance": gr}
    cpu_g = {"albedo": ca, "roughness": cg, "radiance": cr}
    mass = {"albedo": ma, "roughness": mg, "radiance": mr}
    for k in dev_g:
        well = mass[k] <= 10 * np.abs(cpu_g[k])  # conditioning up to 10
        err = np.linalg.norm((dev_g[k] - cpu_g[k])[well]) / np.linalg.norm(cpu_g[k][well])
        print(f"{k}: relative L2 difference {err:.2e} over its {well.sum()} gradients of conditioning up to 10")
        assert err <= 0.01
    pick = np.random.default_rng(64).choice(len(cands), size=min(64, len(cands)), replace=False)
    worst, within1 = 0.0, 0
    for j in pick:
        kind, idx = cands[j]
        g, c, m = dev_g[kind][idx], cpu_g[kind][idx], mass[kind][idx]
        bar = 0.01 * abs(c) + 1e-3 * m + 1e-12
        worst = max(worst, abs(g - c) / bar)
        within1 += abs(g - c) <= 0.01 * abs(c) + 1e-12
        assert abs(g - c) <= bar, (kind, idx, g, c, m)
    print(f"64 parameters: {within1} within 1% of the FP64 value; worst difference {worst:.2f} of its bar")


def test_wavefront_adjoint_matches_plain_replay(field):
    """x2_adjoint (the replay in the wavefront form, credits in the logic and shade kernels) against
    x2_adjoint_plain (one thread a sample): the same samples and the same estimator, so the same gradients up to the
    order of the FP32 partial sums."""
    import torch

    s, scene, albedo, kinds, radiance, roughness = field
    cfg = s.config
    spp = 32
    w = np.random.default_rng(9).random((cfg.width * cfg.height, 3)).astype(np.float32)
    dev = torch.device("cuda", 0)
    dl = torch.from_numpy(w).to(dev)
    scene.set_params(albedo, radiance, roughness)
    out = {}
    for plain in (False, True):
        ga = torch.zeros((len(albedo), 3), dtype=torch.float64, device=dev)
        gr = torch.zeros((len(radiance), 3), dtype=torch.float64, device=dev)
        gg = torch.zeros(len(roughness), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        scene.adjoint(0, spp, dl.data_ptr(), ga.data_ptr(), gr.data_ptr(), gg.data_ptr(), plain=plain)
        out[plain] = [t.cpu().numpy() for t in (ga, gg, gr)]
    for k, name in enumerate(("albedo", "roughness", "radiance")):
        a, b = out[False][k], out[True][k]
        err = np.linalg.norm(a - b) / np.linalg.norm(b)
        print(f"{name}: wavefront vs plain relative L2 {err:.2e}")
        assert err <= 1e-4
        assert np.array_equal(a == 0, b == 0)


def test_texel_gradients(field):
    """dL/dtexel of the heightfield's 64x64 albedo texture: against the FP64 CPU adjoint of the same samples (within 1%
    in L2 over all texels, and 64 seeded random texel channels each within 1% plus 0.1% of the largest) and against
    central differences of single texels (a texel enters its lookups linearly: the bilinear weights of primary hits, the
    closest texel of indirect ones)."""
    import oracle_lib
    import torch

    s, scene, albedo, kinds, radiance, roughness = field
    if not oracle_lib.have_reference():
        pytest.skip("oracle/_ref not built")
    cfg = s.config
    tex = s.texture(0)
    texels = tex.shape[0] * tex.shape[1]
    spp = 16
    w = np.random.default_rng(8).random((cfg.width * cfg.height, 3)).astype(np.float32)
    dev = torch.device("cuda", 0)
    dl = torch.from_numpy(w).to(dev)
    ga = torch.zeros((len(albedo), 3), dtype=torch.float64, device=dev)
    gr = torch.zeros((len(radiance), 3), dtype=torch.float64, device=dev)
    gt = torch.zeros((texels, 3), dtype=torch.float64, device=dev)
    scene.set_params(albedo, radiance, roughness)
    scene.set_texture(0, tex)
    torch.cuda.synchronize()
    scene.adjoint(0, spp, dl.data_ptr(), ga.data_ptr(), gr.data_ptr(), d_texture_grad=gt.data_ptr())
    gt = gt.cpu().numpy()
    ref = oracle_lib.Reference(s)
    *_, tg = oracle_lib.adjoint64(ref, 0, spp, w, params=(albedo, roughness, radiance), texels=texels, texture=tex)
    ref.close()
    err = np.linalg.norm(gt - tg) / np.linalg.norm(tg)
    print(f"texels: relative L2 difference {err:.2e}; nonzero {np.count_nonzero(tg)} of {tg.size}")
    assert err <= 0.01
    live = np.flatnonzero(tg.ravel() != 0)
    pick = np.random.default_rng(65).choice(live, size=min(64, len(live)), replace=False)
    g, c = gt.ravel()[pick], tg.ravel()[pick]
    assert np.all(np.abs(g - c) <= 0.01 * np.abs(c) + 1e-3 * np.abs(tg).max())

    def loss(t):
        scene.set_texture(0, t)
        return float((_image(scene, spp) * w).sum())

    for j in np.argsort(-np.abs(gt.ravel()))[:3]:
        texel, c = divmod(int(j), 3)
        y, x = divmod(texel, tex.shape[1])
        h = 0.02 * tex[y, x, c]
        up, down = tex.copy(), tex.copy()
        up[y, x, c] += h
        down[y, x, c] -= h
        fd = (loss(up) - loss(down)) / (2 * h)
        print(f"texel ({x},{y}) channel {c}: adjoint {gt[texel, c]:.6g} fd {fd:.6g}")
        assert abs(fd - gt[texel, c]) <= 0.03 * abs(gt[texel, c])
    scene.set_texture(0, tex)
