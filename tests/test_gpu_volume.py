"""Participating media (config 3's volume, shrunk: x2_scene_generate 33, a 32^3 grid in the config-0 box, a rect light
and a sun) against the reference's CPU integrator on the same sample identities.

The march's transcendental functions (expf, logf, tanf, atan2f) are the device's own against the host's libm, a few
ulps apart, and a march multiplies dozens of step transmittances; a sample can also take the other branch of a
discrete choice (the step a distance sample picks) when the two sides straddle it. So the bar is a share of samples
within RTOL, every status and alpha alike, and the image within a looser bound.
"""
import numpy as np
import pytest

import oracle_lib
from oracle_lib import x2

pytestmark = pytest.mark.gpu
RTOL, ATOL = 1e-4, 1e-6
needs_reference = pytest.mark.skipif(not oracle_lib.have_reference(), reason="oracle/_ref not built")


@pytest.fixture(scope="module")
def medium(ctx):
    s = x2.SyntheticScene(33)
    return s, x2.Scene(ctx, s.desc, s.config)


@needs_reference
def test_volume_radiance_matches_reference(medium):
    s, scene = medium
    cfg = s.config
    n = cfg.width * cfg.height
    px = np.arange(n, dtype=np.uint32)
    idx = np.full(n, 2, np.uint32)
    rgba, status = scene.integrate(px, idx)
    rrgba, rstatus = oracle_lib.Reference(s).integrate(px, idx)
    assert np.array_equal(status, rstatus)
    ok = (np.abs(rgba - rrgba) <= RTOL * np.abs(rrgba) + ATOL).all(axis=1)
    print(f"volume: {ok.mean() * 100:.3f}% of {n} samples within {RTOL}")
    assert ok.mean() >= 0.99
    assert np.allclose(rgba[:, :3].mean(axis=0), rrgba[:, :3].mean(axis=0), rtol=2e-3)
    assert np.allclose(rgba[:, 3], rrgba[:, 3], rtol=1e-3, atol=1e-5)


@needs_reference
def test_volume_changes_the_image(medium):
    """The medium is there: the same samples without it differ (darker walls through it, its glow and in-scattering)."""
    s, scene = medium
    cfg = s.config
    n = cfg.width * cfg.height
    px = np.arange(n, dtype=np.uint32)
    idx = np.zeros(n, np.uint32)
    with_volume, _ = scene.integrate(px, idx)
    bare = x2.SyntheticScene(33)
    bare_cfg = bare.config
    bare_cfg.volume_count = 0
    ref = oracle_lib.Reference(bare, bare_cfg)
    without, _ = ref.integrate(px, idx)
    assert np.abs(with_volume[:, :3] - without[:, :3]).mean() > 1e-3


def test_volume_wavefront_equals_plain(medium):
    s, scene = medium
    spp = s.config.spp
    scene.frame_begin(spp)
    scene.render_frame(0, spp)
    scene.wait()
    scene.audit()
    plain, pc = scene.film()
    scene.frame_begin(spp)
    scene.render_frame_wavefront(0, spp)
    scene.wait()
    scene.audit()
    wave, wc = scene.film()
    assert np.array_equal(pc, wc)
    assert np.allclose(plain, wave, rtol=1e-12, atol=1e-12)


def test_volume_configs_refused(ctx, medium):
    s, scene = medium
    cfg = x2.Config.from_buffer_copy(s.config)
    cfg.max_volume_depth = 65
    with pytest.raises(x2.X2Error) as e:
        scene.set_config(cfg)
    assert e.value.code == x2.EINVAL
    scene.set_config(s.config)


def _multiple(s, depth):
    cfg = x2.Config.from_buffer_copy(s.config)
    cfg.max_volume_depth = depth
    cfg.volume_illumination_samples = 2
    return cfg


@needs_reference
@pytest.mark.parametrize("depth", [2, 4])
def test_multiple_scattering_matches_reference(medium, depth):
    """The multiple-scattering approximation (max_volume_depth above one: free paths from scatter events, each order's
    light through its attenuation and contribution factors) against the reference's on the same identities."""
    s, scene = medium
    cfg = _multiple(s, depth)
    scene.set_config(cfg)
    try:
        n = cfg.width * cfg.height
        px = np.arange(n, dtype=np.uint32)
        idx = np.full(n, 3, np.uint32)
        rgba, status = scene.integrate(px, idx)
        rrgba, rstatus = oracle_lib.Reference(s, cfg).integrate(px, idx)
        single = oracle_lib.Reference(s, s.config).integrate(px, idx)[0]
    finally:
        scene.set_config(s.config)
    assert np.array_equal(status, rstatus)
    ok = (np.abs(rgba - rrgba) <= RTOL * np.abs(rrgba) + ATOL).all(axis=1)
    print(f"multiple scattering, depth {depth}: {ok.mean() * 100:.3f}% of {n} samples within {RTOL}; "
          f"mean {rgba[:, :3].mean():.6f} against single scattering's {single[:, :3].mean():.6f}")
    assert ok.mean() >= 0.99
    assert np.allclose(rgba[:, :3].mean(axis=0), rrgba[:, :3].mean(axis=0), rtol=2e-3)
    assert rrgba[:, :3].mean() > single[:, :3].mean()  # the higher orders add light


def test_multiple_scattering_wavefront_equals_plain(medium):
    s, scene = medium
    cfg = _multiple(s, 3)
    scene.set_config(cfg)
    try:
        spp = 4
        scene.frame_begin(spp)
        scene.render_frame(0, spp)
        scene.wait()
        plain, pc = scene.film()
        scene.frame_begin(spp)
        scene.render_frame_wavefront(0, spp)
        scene.wait()
        wave, wc = scene.film()
    finally:
        scene.set_config(s.config)
    assert np.array_equal(pc, wc)
    assert np.allclose(plain, wave, rtol=1e-12, atol=1e-12)


def test_volume_golden(medium):
    """The committed golden radiance of the reference on this scene (no reference build needed on the device box)."""
    import os

    s, scene = medium
    g = np.load(os.path.join(oracle_lib.ROOT, "tests", "golden", "radiance_c33.npz"))
    rgba, status = scene.integrate(g["pixels"], g["indices"])
    assert np.array_equal(status, g["status"])
    ok = (np.abs(rgba - g["rgba"]) <= RTOL * np.abs(g["rgba"]) + ATOL).all(axis=1)
    print(f"volume golden: {ok.mean() * 100:.3f}% of {len(ok)} samples within {RTOL}")
    assert ok.mean() >= 0.99
