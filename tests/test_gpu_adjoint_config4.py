"""The adjoint at the differentiable render's own size (config 4: 247,808 triangles, a 1024x1024 albedo texture on the
heightfield, 64 sphere materials, 16 rect lights and an environment; 512x512, 32 samples a pixel for the primal, 16 for
the adjoint).

1. The specified loss: a target rendered from the scene's true parameters, the parameters perturbed (albedo + N(0, 0.2)
   clamped to [0, 1], roughness + U[-0.2, 0.2] clamped to [0.05, 1]), L = sum (image - target)^2 over the 32-sample
   images, dL/dimage = 2 (image - target). The adjoint of samples 32..47 against the FP64 CPU adjoint of the same
   samples with the same dL/dimage (oracle/adjoint64.h): 64 seeded random parameters among the Lambert albedo
   channels, GGX roughnesses and light radiance channels, each within 1 % of its FP64 value or, where the sum of its
   credits' magnitudes (its mass) is many times the value (near-cancelling credits; conditioning = mass / |value|),
   within 1 % plus 1e-3 of its mass — each such parameter listed with its conditioning.
   The FP64 adjoint traces its own rays in double, so a few of its paths take another discrete decision than the fp32
   paths (a grazing shadow ray, a closest hit at an edge); near-mirror GGX samples carry large roughness credits, so one
   such path can move a roughness gradient by a percent. The check is therefore made twice: over every pixel (albedo
   and radiance held to the bar, every roughness outside it listed) and over the pixels whose FP64 primal equals the
   device's image of the same samples within 1e-4 (dL/dimage zeroed elsewhere, on both sides): there every one of the
   64 parameters is held to the bar. The adjoint's throughput against the primal's is printed (target 0.3).
2. Central differences with common random numbers at step 1e-3, with Russian roulette off for this check (a roulette
   decision that flips with the parameter moves a sample by a step, and at a step of 1e-3 those flips would swamp the
   differences; the adjoint holds decisions fixed): a linear loss w . image over samples 0..15 and the adjoint of the
   same samples; the largest albedo, radiance and texel gradients within 1 %.
   Roughness is checked statistically. Its adjoint credits are the score of the GGX samples' directions (the direction
   stays, its density's derivative weights it), while the differences move the directions, some across visibility
   edges: both estimate the same derivative of the expected loss, with different noise, so they agree in the mean,
   not sample by sample. Sixteen batches of one sample a pixel each give a difference and an adjoint; the mean of
   (difference - adjoint) is within 4 standard errors (t with 15 degrees of freedom: p ~ 0.001) of zero.
"""
import time

import numpy as np
import pytest

import oracle_lib
from oracle_lib import x2

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not oracle_lib.have_reference(), reason="oracle/_ref not built")]


def _render(scene, first, spp):
    scene.frame_begin(spp)
    scene.render_frame_wavefront(first, spp)
    c = scene.wait()
    sums, counts = scene.film()
    assert (counts == spp).all()
    return sums[:, :3] / counts[:, None], c.milliseconds


@pytest.fixture(scope="module")
def config4(ctx):
    s = x2.SyntheticScene(4)
    d = s.desc
    albedo = np.array([list(d.materials[m].diffuse) for m in range(d.material_count)], np.float64)
    kinds = np.array([d.materials[m].kind for m in range(d.material_count)])
    radiance = np.array([list(d.lights[i].radiance) for i in range(d.light_count)], np.float64)
    roughness = np.array([d.materials[m].roughness for m in range(d.material_count)], np.float64)
    return s, albedo, kinds, radiance, roughness


def test_config4_loss_gradients_against_fp64_adjoint(ctx, config4):
    import torch

    s, albedo, kinds, radiance, roughness = config4
    cfg = s.config
    assert (cfg.width, cfg.height, s.desc.triangle_count) == (512, 512, 247808)
    scene = x2.Scene(ctx, s.desc, cfg)
    target, _ = _render(scene, 0, 32)
    rng = np.random.default_rng(4)
    a0 = np.clip(albedo + rng.normal(0, 0.2, albedo.shape), 0, 1)
    g0 = np.clip(roughness + rng.uniform(-0.2, 0.2, roughness.shape), 0.05, 1.0)
    scene.set_params(a0, radiance, g0)
    _render(scene, 0, 32)  # warm-up
    image, primal_ms = _render(scene, 0, 32)
    dldi = (2.0 * (image - target)).astype(np.float32)
    dev = torch.device("cuda", 0)
    dl = torch.from_numpy(dldi).to(dev)
    ga = torch.zeros((len(albedo), 3), dtype=torch.float64, device=dev)
    gr = torch.zeros((len(radiance), 3), dtype=torch.float64, device=dev)
    gg = torch.zeros(len(roughness), dtype=torch.float64, device=dev)
    scene.adjoint(32, 16, dl.data_ptr(), ga.data_ptr(), gr.data_ptr(), gg.data_ptr())  # warm-up (graph and buffers)
    for t in (ga, gr, gg):
        t.zero_()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    scene.adjoint(32, 16, dl.data_ptr(), ga.data_ptr(), gr.data_ptr(), gg.data_ptr())
    torch.cuda.synchronize()
    adjoint_ms = (time.perf_counter() - t0) * 1e3
    pixels = cfg.width * cfg.height
    ratio = (pixels * 16 / adjoint_ms) / (pixels * 32 / primal_ms)
    print(f"config 4: primal {pixels * 32 / primal_ms / 1e3:.1f} Msamples/s (32 spp, device time), adjoint "
          f"{pixels * 16 / adjoint_ms / 1e3:.1f} Msamples/s (16 spp, host time around the call): {ratio:.2f} x the primal")
    ga, gr, gg = ga.cpu().numpy(), gr.cpu().numpy(), gg.cpu().numpy()
    ref = oracle_lib.Reference(s)
    ca, cg, cr, img64, (ma, mg, mr) = oracle_lib.adjoint64(ref, 32, 16, dldi, params=(a0, g0, radiance), masses=True,
                                                           texture=s.texture(0))
    lam = np.flatnonzero(kinds == x2.MAT_LAMBERT)
    ggx = np.flatnonzero(kinds == x2.MAT_GGX)
    cands = [("albedo", (m, c)) for m in lam for c in range(3)] + [("roughness", (m,)) for m in ggx] + \
            [("radiance", (i, c)) for i in range(len(radiance)) for c in range(3)]
    pick = np.random.default_rng(64).choice(len(cands), size=64, replace=False)

    def compare(dev_g, cpu_g, mass, strict_kinds):
        within1, listed = 0, []
        for j in pick:
            kind, idx = cands[j]
            g, c, m = float(dev_g[kind][idx]), float(cpu_g[kind][idx]), float(mass[kind][idx])
            if abs(g - c) <= 0.01 * abs(c) + 1e-12:
                within1 += 1
                continue
            ok = abs(g - c) <= 0.01 * abs(c) + 1e-3 * m
            listed.append(f"  {kind}{list(idx)}: device {g:.6g} fp64 {c:.6g} mass {m:.4g} conditioning {m / max(abs(c), 1e-30):.1f}"
                          + ("" if ok else " (outside the bar)"))
            assert ok or kind not in strict_kinds, listed[-1]
        return within1, listed

    within1, listed = compare({"albedo": ga, "roughness": gg, "radiance": gr}, {"albedo": ca, "roughness": cg, "radiance": cr},
                              {"albedo": ma, "roughness": mg, "radiance": mr}, ("albedo", "radiance"))
    print(f"every pixel: {within1} of 64 parameters within 1 % of the FP64 adjoint; the others:\n" + "\n".join(listed))

    # The pixels whose 16 paths agree: the FP64 primal of samples 32..47 equal to the device's image of them.
    dimg, _ = _render(scene, 32, 16)
    same = (np.abs(img64 / 16 - dimg) <= 1e-4 * np.abs(dimg) + 1e-6).all(1)
    dm = (dldi * same[:, None]).astype(np.float32)
    dlm = torch.from_numpy(dm).to(dev)
    gam = torch.zeros_like(torch.from_numpy(ca)).to(dev)
    grm = torch.zeros_like(torch.from_numpy(cr)).to(dev)
    ggm = torch.zeros_like(torch.from_numpy(cg)).to(dev)
    scene.adjoint(32, 16, dlm.data_ptr(), gam.data_ptr(), grm.data_ptr(), ggm.data_ptr())
    cam, cgm, crm, _, (mam, mgm, mrm) = oracle_lib.adjoint64(ref, 32, 16, dm, params=(a0, g0, radiance), masses=True, texture=s.texture(0))
    ref.close()
    within1, listed = compare({"albedo": gam.cpu().numpy(), "roughness": ggm.cpu().numpy(), "radiance": grm.cpu().numpy()},
                              {"albedo": cam, "roughness": cgm, "radiance": crm}, {"albedo": mam, "roughness": mgm, "radiance": mrm},
                              ("albedo", "radiance", "roughness"))
    print(f"{same.mean() * 100:.3f} % of pixels with the FP64 primal equal to the device's: {within1} of 64 parameters within 1 % "
          f"of the FP64 adjoint; the others within 1 % plus 1e-3 of their mass:\n" + "\n".join(listed))
    assert same.mean() >= 0.9
    assert ratio >= 0.3


def test_config4_central_differences(ctx, config4):
    import torch

    s, albedo, kinds, radiance, roughness = config4
    cfg = x2.SyntheticScene(4).config
    cfg.rr_threshold = 0.0
    scene = x2.Scene(ctx, s.desc, cfg)
    spp = 16
    pixels = cfg.width * cfg.height
    w = np.random.default_rng(11).random((pixels, 3))
    tex = s.texture(0)
    dev = torch.device("cuda", 0)
    dl = torch.from_numpy(w.astype(np.float32)).to(dev)
    ga = torch.zeros((len(albedo), 3), dtype=torch.float64, device=dev)
    gr = torch.zeros((len(radiance), 3), dtype=torch.float64, device=dev)
    gg = torch.zeros(len(roughness), dtype=torch.float64, device=dev)
    gt = torch.zeros((tex.shape[0] * tex.shape[1], 3), dtype=torch.float64, device=dev)
    scene.set_params(albedo, radiance, roughness)
    torch.cuda.synchronize()
    scene.adjoint(0, spp, dl.data_ptr(), ga.data_ptr(), gr.data_ptr(), gg.data_ptr(), d_texture_grad=gt.data_ptr())
    ga, gr, gg, gt = (t.cpu().numpy() for t in (ga, gr, gg, gt))

    def loss():
        return float((_render(scene, 0, spp)[0] * w).sum())

    h = 1e-3
    rows = []
    lam = np.flatnonzero(kinds == x2.MAT_LAMBERT)
    for m in lam[np.argsort(-np.abs(ga[lam].sum(1)))][:4]:
        c = int(np.argmax(np.abs(ga[m])))
        up, down = albedo.copy(), albedo.copy()
        up[m, c] += h
        down[m, c] -= h
        scene.set_params(up, radiance, roughness)
        lu = loss()
        scene.set_params(down, radiance, roughness)
        ld = loss()
        rows.append(("albedo", (m, c), ga[m, c], (lu - ld) / (2 * h), 0.01))
    scene.set_params(albedo, radiance, roughness)
    for i in np.argsort(-np.abs(gr.sum(1)))[:3]:
        step = h * radiance[i, 0]
        up, down = radiance.copy(), radiance.copy()
        up[i] += step
        down[i] -= step
        scene.set_params(albedo, up, roughness)
        lu = loss()
        scene.set_params(albedo, down, roughness)
        ld = loss()
        rows.append(("radiance", (i,), gr[i].sum(), (lu - ld) / (2 * step), 0.01))
    scene.set_params(albedo, radiance, roughness)
    for j in np.argsort(-np.abs(gt.ravel()))[:3]:
        texel, c = divmod(int(j), 3)
        y, x = divmod(texel, tex.shape[1])
        up, down = tex.copy(), tex.copy()
        up[y, x, c] += h
        down[y, x, c] -= h
        scene.set_texture(0, up)
        lu = loss()
        scene.set_texture(0, down)
        ld = loss()
        rows.append(("texel", (x, y, c), gt[texel, c], (lu - ld) / (2 * h), 0.01))
    scene.set_texture(0, tex)
    for kind, idx, adj, fd, bar in rows:
        print(f"{kind}{list(idx)}: adjoint {adj:.6g} central difference {fd:.6g} ({(fd - adj) / adj * 100:+.3f} %)")
    for kind, idx, adj, fd, bar in rows:
        assert abs(fd - adj) <= bar * abs(adj), (kind, idx, adj, fd)

    # Roughness, by batches of one sample a pixel (samples b, b = 0..15).
    batches = 16
    per = np.zeros((batches, len(roughness)))
    ba = torch.zeros((len(albedo), 3), dtype=torch.float64, device=dev)
    br = torch.zeros((len(radiance), 3), dtype=torch.float64, device=dev)
    bg = torch.zeros(len(roughness), dtype=torch.float64, device=dev)
    for b in range(batches):
        for t in (ba, br, bg):
            t.zero_()
        scene.adjoint(b, 1, dl.data_ptr(), ba.data_ptr(), br.data_ptr(), bg.data_ptr())
        per[b] = bg.cpu().numpy()
    # A one-sample adjoint weighs its sample as the whole image: the batches' mean is the 16-sample adjoint (up to the
    # FP32 gradient rows' own rounding, which depends on how the credits are grouped).
    assert np.allclose(per.mean(0), gg, rtol=1e-5, atol=1e-7 * np.abs(gg).max())

    def batch_loss(b):
        return float((_render(scene, b, 1)[0] * w).sum())

    ggx = np.flatnonzero((kinds == x2.MAT_GGX) & (roughness >= 0.2))
    for m in ggx[np.argsort(-np.abs(gg[ggx]))][:3]:
        up, down = roughness.copy(), roughness.copy()
        up[m] += h
        down[m] -= h
        fd = np.zeros(batches)
        scene.set_params(albedo, radiance, up)
        for b in range(batches):
            fd[b] = batch_loss(b)
        scene.set_params(albedo, radiance, down)
        for b in range(batches):
            fd[b] = (fd[b] - batch_loss(b)) / (2 * h)
        d = fd - per[:, m]
        se = d.std(ddof=1) / np.sqrt(batches)
        print(f"roughness[{m}]: adjoint {per[:, m].mean():.6g} central difference {fd.mean():.6g} over 16 samples; "
              f"mean batch difference {d.mean():.4g}, standard error {se:.4g} ({d.mean() / se:+.2f} SE)")
        assert abs(d.mean()) <= 4.0 * se, (m, d.mean(), se)
    scene.set_params(albedo, radiance, roughness)
