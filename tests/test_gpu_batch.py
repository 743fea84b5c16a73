"""Batched renders (x2_render_batch): many scenes of uneven resolution, spp and depth in one wavefront launch.

Each request's film must be exactly the film the single-scene wavefront launch gives for the same samples (the same
per-sample arithmetic and the same sample-order film sums), agree with the plain megakernel's film to FP64 summation
order, and pass the sample-count audit. The requests are config 2's, shrunk (x2_scene_generate 300 + r).
"""
import numpy as np
import pytest

from oracle_lib import x2

pytestmark = pytest.mark.gpu

REQUESTS = list(range(300, 308))


def _scenes(ctx, ids):
    out = []
    for i in ids:
        s = x2.SyntheticScene(i)
        out.append((s, x2.Scene(ctx, s.desc, s.config)))
    return out


def _single_wavefront_film(scene, first, count):
    cfg = scene.config
    tiles = ((cfg.width + 7) // 8) * ((cfg.height + 7) // 8)
    chunks = np.zeros(tiles, x2.CHUNK_DTYPE)
    chunks["tile"], chunks["first"], chunks["count"] = np.arange(tiles), first, count
    scene.frame_begin(count)
    scene.launch_wavefront(chunks)
    scene.wait()
    scene.audit()
    return scene.film()


@pytest.mark.parametrize("window", [0, 4096])
def test_batch_films_equal_single_launches(ctx, window):
    scenes = _scenes(ctx, REQUESTS)
    scenes[0][1].wavefront_tune(batch_window=window)
    requests = [(sc, 3 * k, s.config.spp) for k, (s, sc) in enumerate(scenes)]
    done = ctx.render_batch(requests)
    expected = sum(s.config.width * s.config.height * s.config.spp for s, _ in scenes)
    assert done.samples == expected and done.errors == 0
    batch = []
    for (s, sc), (_, first, count) in zip(scenes, requests):
        sc.audit()
        batch.append(sc.film())
    for (s, sc), (_, first, count), (bsums, bcounts) in zip(scenes, requests, batch):
        sums, counts = _single_wavefront_film(sc, first, count)
        assert np.array_equal(bcounts, counts), s.config_id
        assert np.array_equal(bsums, sums), s.config_id


def test_batch_agrees_with_plain_megakernel(ctx):
    scenes = _scenes(ctx, REQUESTS[:4])
    requests = [(sc, 0, s.config.spp) for s, sc in scenes]
    ctx.render_batch(requests)
    batch = [sc.film() for _, sc in scenes]
    for (s, sc), (bsums, bcounts) in zip(scenes, batch):
        sc.frame_begin(s.config.spp)
        sc.render_frame(0, s.config.spp)
        sc.wait()
        sc.audit()
        sums, counts = sc.film()
        assert np.array_equal(bcounts, counts)
        assert np.allclose(bsums, sums, rtol=1e-12, atol=1e-12)


def test_batch_rejects_bad_requests(ctx):
    (s0, a), (s1, b) = _scenes(ctx, REQUESTS[:2])
    with pytest.raises(x2.X2Error) as e:
        ctx.render_batch([(a, 0, 1), (a, 1, 1)])
    assert e.value.code == x2.EINVAL
    cfg = s1.config
    cfg.bsdf_samples = 2
    b.set_config(cfg)
    with pytest.raises(x2.X2Error) as e:
        ctx.render_batch([(a, 0, 1), (b, 0, 1)])
    assert e.value.code == x2.EINVAL
