"""Delta and ratio tracking over majorant grids (x2_config.volume_estimator = 1): a second estimator of the volume
integrals the reference's decoupled march estimates, so it has no per-sample parity with the reference; it is judged
against the reference's converged render of the participating medium (config 3; tests/golden/rmse_c3.npz: 16,384
samples a pixel of the reference's march, FP64 film).

Bar: each fixture pixel's mean over 4,096 tracked samples against the converged value, in units of the combined
standard error (the tracked mean's, from the samples' own variance, and the reference's, its variance over 16,384):
the z-scores' root mean square at most 1.5 (1 for an unbiased estimator whose only difference is noise; the march's own
quadrature, which the reference image carries, is the rest), and the image means within 1 % of each other.
"""
import os

import numpy as np
import pytest

import rmse_lib
from oracle_lib import x2

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_tracking_converges_to_the_reference(ctx):
    f = np.load(os.path.join(GOLDEN, "rmse_c3.npz"))
    s = x2.SyntheticScene(3)
    cfg = s.config
    cfg.volume_estimator = 1
    scene = x2.Scene(ctx, s.desc, cfg)
    px = rmse_lib.tile_pixels(f["tiles"], cfg.width, cfg.height)
    live = f["live"]
    pixels = px[live].astype(np.uint32)
    n = 4096
    sums = np.zeros((len(pixels), 3))
    squares = np.zeros((len(pixels), 3))
    for first in range(0, n, 1024):
        p = np.repeat(pixels, 1024)
        idx = np.tile(np.arange(first, first + 1024, dtype=np.uint32), len(pixels))
        rgba, status = scene.integrate(p, idx)
        assert (status == x2.DONE).all()
        v = rgba[:, :3].reshape(len(pixels), 1024, 3)
        sums += v.sum(1)
        squares += (v ** 2).sum(1)
    mean = sums / n
    var = np.maximum(squares / n - mean ** 2, 0.0) * n / (n - 1)
    ref = f["ref"][live].astype(np.float64)
    se = np.sqrt(var / n + var / 16384 + 1e-12)
    z = (mean - ref) / se
    rms = float(np.sqrt(np.mean(z ** 2)))
    rel = float(mean.mean() / ref.mean() - 1.0)
    print(f"tracking: {len(pixels)} pixels x {n} samples; z rms {rms:.3f}, mean z {z.mean():.3f}, image mean {mean.mean():.6f} against "
          f"{ref.mean():.6f} ({rel * 100:+.3f} %)")
    assert rms <= 1.5
    assert abs(rel) <= 0.01


def _fixture_means(scene, pixels, n):
    sums = np.zeros((len(pixels), 3))
    for first in range(0, n, 1024):
        p = np.repeat(pixels, 1024)
        idx = np.tile(np.arange(first, first + 1024, dtype=np.uint32), len(pixels))
        rgba, status = scene.integrate(p, idx)
        assert (status == x2.DONE).all()
        sums += rgba[:, :3].reshape(len(pixels), 1024, 3).sum(1)
    return sums / n


def test_tracking_is_the_limit_of_finer_marches(ctx):
    """The march is a quadrature: its step (the least feature size times inv_volume_quality) carries a bias that
    tracking, which samples the continuous density, does not. With the steps 4 and 16 times finer, the march's image
    mean moves toward the tracked one: the gap shrinks, and at 16 times finer it is within 0.3 % (tracked over 16,384
    samples a pixel and marched over 4,096, the two means' standard errors are under 0.1 % each)."""
    f = np.load(os.path.join(GOLDEN, "rmse_c3.npz"))
    s = x2.SyntheticScene(3)
    pixels = rmse_lib.tile_pixels(f["tiles"], s.config.width, s.config.height)[f["live"]].astype(np.uint32)

    def image_mean(estimator, finer, n):
        cfg = x2.SyntheticScene(3).config
        cfg.volume_estimator = estimator
        cfg.inv_volume_quality /= finer
        cfg.inv_volume_shadow_quality /= finer
        scene = x2.Scene(ctx, s.desc, cfg)
        m = float(_fixture_means(scene, pixels, n).mean())
        scene.free()
        return m

    tracked = image_mean(1, 1, 16384)
    gaps = {k: image_mean(0, k, 4096) / tracked - 1.0 for k in (1, 4, 16)}
    print(f"tracking image mean {tracked:.6f}; the march's relative to it at steps 1, 1/4, 1/16: "
          + ", ".join(f"{g * 100:+.3f} %" for g in gaps.values()))
    assert abs(gaps[16]) < abs(gaps[1])
    assert abs(gaps[16]) <= 0.003


def test_tracking_refuses_unadmitted_configs(ctx):
    s = x2.SyntheticScene(3)
    for field, value in (("max_volume_depth", 2), ("volume_overlap_mode", 2), ("volume_estimator", 2)):
        cfg = x2.SyntheticScene(3).config
        cfg.volume_estimator = 1
        setattr(cfg, field, value)
        with pytest.raises(x2.X2Error) as e:
            x2.Scene(ctx, s.desc, cfg)
        assert e.value.code == x2.EINVAL, field
