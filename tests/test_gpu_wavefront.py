"""GPU tests of the wavefront form: the same samples as the plain megakernel (per item, per pixel, per count), whatever
the number of paths in flight; the reference's order of contributions is kept, so per-sample radiance is identical."""
import numpy as np
import pytest

import oracle_lib
from oracle_lib import x2

pytestmark = pytest.mark.gpu


def items_of(cfg, chunks, spc):
    """(pixel, index) of every item of a launch, and whether it is a sample (item order of the lane API)."""
    tiles_x = (cfg.width + 7) // 8
    pix, idx, valid = [], [], []
    for c in chunks:
        for pos in range(64):
            for s in range(spc):
                x = (c["tile"] % tiles_x) * 8 + pos % 8
                y = (c["tile"] // tiles_x) * 8 + pos // 8
                ok = s < c["count"] and x < cfg.width and y < cfg.height
                pix.append(y * cfg.width + x if ok else 0)
                idx.append(c["first"] + s)
                valid.append(ok)
    return np.array(pix, np.uint32), np.array(idx, np.uint32), np.array(valid)


@pytest.mark.parametrize("cid,paths", [(0, 0), (108, 0), (108, 1024)])
def test_wavefront_items_equal_plain_samples(ctx, cid, paths):
    s = x2.SyntheticScene(cid)
    scene = x2.Scene(ctx, s.desc, s.config)
    cfg = s.config
    tiles = ((cfg.width + 7) // 8) * ((cfg.height + 7) // 8)
    r = np.random.default_rng(cid + paths)
    sel = np.sort(r.choice(tiles, size=min(tiles, 40), replace=False))
    spc = 6
    chunks = np.zeros(len(sel), x2.CHUNK_DTYPE)
    chunks["tile"], chunks["first"], chunks["count"] = sel, r.integers(0, 50, len(sel)), r.integers(1, spc + 1, len(sel))
    if paths:
        scene.wavefront_reserve(paths)
    scene.frame_begin(spc)
    scene.launch_wavefront(chunks)
    c = scene.wait()
    assert c.errors == 0
    px, idx, valid = items_of(cfg, chunks, spc)
    rgba, status = scene.items(len(px))
    assert (status[~valid] == x2.SKIP).all()
    assert (status[valid] == x2.DONE).all()
    want, wstatus = scene.integrate(px[valid], idx[valid])
    assert (wstatus == x2.DONE).all()
    got = rgba[valid].astype(np.float64)
    assert np.array_equal(got, want), f"max abs diff {np.abs(got - want).max()}"
    sums, counts = scene.film()
    # The film is the per-pixel sum of the launch's samples.
    expect = np.zeros((cfg.width * cfg.height, 4))
    np.add.at(expect, px[valid], want)
    cnt = np.bincount(px[valid], minlength=cfg.width * cfg.height)
    assert np.array_equal(counts, cnt)
    assert np.allclose(sums, expect, rtol=1e-12, atol=1e-12)
    info = scene.wavefront_info()
    assert info["records_per_path"] == cfg.light_count * cfg.light_samples + 1
    assert scene.counters()["stack_overflows"] == 0


def test_wavefront_frame_matches_plain_frame(ctx):
    s = x2.SyntheticScene(108)
    cfg = s.config
    cfg.spp = 4
    scene = x2.Scene(ctx, s.desc, cfg)
    scene.frame_begin(4)
    scene.render_frame(0, 4)
    scene.wait()
    scene.audit()
    plain, pc = scene.film()
    pcount = scene.counters()
    scene.reset_counters()
    scene.frame_begin(4)
    scene.render_frame_wavefront(0, 4)
    scene.wait()
    scene.audit()
    wave, wc = scene.film()
    wcount = scene.counters()
    assert np.array_equal(pc, wc)
    assert np.allclose(plain, wave, rtol=1e-12, atol=1e-12)
    for k in ("trace", "shadow_nee", "shadow_bsdf", "held", "samples"):
        assert pcount[k] == wcount[k], k


def test_wavefront_rejects_many_bsdf_samples(ctx):
    s = x2.SyntheticScene(0)
    cfg = s.config
    cfg.bsdf_samples = 2
    scene = x2.Scene(ctx, s.desc, cfg)
    scene.frame_begin(1)
    with pytest.raises(x2.X2Error) as e:
        scene.render_frame_wavefront(0, 1)
    assert e.value.code == x2.EINVAL


def test_autotuned_shape_renders_the_same_film(ctx):
    s = x2.SyntheticScene(108)
    cfg = s.config
    cfg.spp = 4
    scene = x2.Scene(ctx, s.desc, cfg)
    scene.frame_begin(4)
    scene.render_frame_wavefront(0, 4)
    scene.wait()
    want, wc = scene.film()
    shape, ms = scene.wavefront_autotune(tiles=64, spp=4)
    assert ms > 0 and 1 <= shape["refill"] <= 32 and 1 <= shape["tri_limit"] <= 32
    scene.frame_begin(4)
    scene.render_frame_wavefront(0, 4)
    scene.wait()
    scene.audit()
    got, gc = scene.film()
    assert np.array_equal(gc, wc)
    assert np.array_equal(got, want)


SHAPES = [{"shadow_order": 1}, {"extend_bins": 1}, {"blocks_per_sm": 16}, {"short_stack": 0}, {"trace_blocks": 9}, {"lobe_queues": 0},
          {"shade_split": 0}, {"light_split": 0}, {"tri_limit": 3}, {"refill": 1}, {"paths": 1024}, {"shade_blocks": 3},
          {"shadow_order": 1, "light_split": 1}, {"tri_overlap": 0}, {"tri_overlap": 0, "shadow_order": 1}]


@pytest.mark.parametrize("shape", SHAPES, ids=lambda d: ",".join(f"{k}={v}" for k, v in d.items()))
def test_every_launch_shape_renders_the_same_film(ctx, shape):
    """The launch shape moves work between lanes, queues and steps, never the samples' arithmetic: the film and the
    counters equal the default shape's bit for bit (config 108: GGX and Lambert, 16 rect lights and an environment)."""
    s = x2.SyntheticScene(108)
    cfg = s.config
    cfg.spp = 4
    scene = x2.Scene(ctx, s.desc, cfg)
    scene.frame_begin(4)
    scene.render_frame_wavefront(0, 4)
    scene.wait()
    want, wc = scene.film()
    base = scene.counters()
    scene.reset_counters()
    scene.wavefront_tune(**shape)
    scene.frame_begin(4)
    scene.render_frame_wavefront(0, 4)
    scene.wait()
    scene.audit()
    got, gc = scene.film()
    assert np.array_equal(gc, wc)
    assert np.array_equal(got, want)
    after = scene.counters()
    for k in ("trace", "shadow_nee", "shadow_bsdf", "held", "samples", "errors", "stack_overflows"):
        assert after[k] == base[k], k
