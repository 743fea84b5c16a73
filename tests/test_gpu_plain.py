"""GPU tests of the plain megakernel's frame launch (x2_launch): per sample, the film holds exactly the radiance the
per-sample entry (x2_integrate, one thread a sample) gives for the same identity, and the launch's counters are the
wavefront form's. Surface scenes whose vertices make at most 24 shadow rays run the bounce-at-a-time kernel
(renderSteps), the others (volume scenes among them) the one-thread-a-sample kernel (renderChunks); both must meet the
same bar."""
import numpy as np
import pytest

from oracle_lib import x2

pytestmark = pytest.mark.gpu


def one_sample_chunks(cfg, n_tiles, seed):
    """Distinct random tiles, each pixel of a tile taking one sample of a random index."""
    tiles = ((cfg.width + 7) // 8) * ((cfg.height + 7) // 8)
    r = np.random.default_rng(seed)
    sel = np.sort(r.choice(tiles, size=min(tiles, n_tiles), replace=False))
    chunks = np.zeros(len(sel), x2.CHUNK_DTYPE)
    chunks["tile"], chunks["first"], chunks["count"] = sel, r.integers(0, 4096, len(sel)), 1
    return chunks


def tile_pixels(cfg, tile):
    tiles_x = (cfg.width + 7) // 8
    out = []
    for pos in range(64):
        x, y = (tile % tiles_x) * 8 + pos % 8, (tile // tiles_x) * 8 + pos // 8
        if x < cfg.width and y < cfg.height:
            out.append(y * cfg.width + x)
    return out


@pytest.mark.parametrize("cid", [0, 108, 44, 33])
def test_plain_frame_sample_equals_per_sample_entry(ctx, cid):
    """One sample a pixel: the film's FP64 sum is that sample's float radiance, so it must equal x2_integrate's bit
    for bit (config 0: the closed box; 108: GGX and Lambert under 16 rect lights and an environment; 44: the textured
    heightfield; 33: the participating medium in the box, one thread a sample)."""
    s = x2.SyntheticScene(cid)
    cfg = s.config
    scene = x2.Scene(ctx, s.desc, cfg)
    chunks = one_sample_chunks(cfg, 300, cid)
    scene.frame_begin(1)
    scene.launch(chunks)
    c = scene.wait()
    assert c.errors == 0
    px, idx = [], []
    for ch in chunks:
        p = tile_pixels(cfg, int(ch["tile"]))
        px += p
        idx += [int(ch["first"])] * len(p)
    px, idx = np.array(px, np.uint32), np.array(idx, np.uint32)
    want, status = scene.integrate(px, idx)
    assert (status == x2.DONE).all()
    sums, counts = scene.film()
    assert counts.sum() == len(px) and (counts[px] == 1).all()
    got = sums[px]
    bad = np.flatnonzero((got != want).any(axis=1))
    assert bad.size == 0, f"{bad.size} of {len(px)} samples differ, first pixel {px[bad[0]]}: {got[bad[0]]} vs {want[bad[0]]}"
    scene.free()


@pytest.mark.parametrize("cid", [108, 44, 33])
def test_plain_launch_counts_the_wavefront_rays(ctx, cid):
    """Ragged chunks (1..6 samples a pixel, edge tiles included): the same film as the wavefront form to FP64 summation
    order, the same counts, and the same rays (closest, light-sample and BSDF shadow rays, held lights, samples)."""
    s = x2.SyntheticScene(cid)
    cfg = s.config
    scene = x2.Scene(ctx, s.desc, cfg)
    tiles = ((cfg.width + 7) // 8) * ((cfg.height + 7) // 8)
    r = np.random.default_rng(7 + cid)
    sel = np.unique(np.concatenate([r.choice(tiles, min(tiles, 120), replace=False), [tiles - 1]]))
    chunks = np.zeros(len(sel), x2.CHUNK_DTYPE)
    chunks["tile"], chunks["first"], chunks["count"] = sel, r.integers(0, 100, len(sel)), r.integers(1, 7, len(sel))
    out = {}
    for form in ("plain", "wavefront"):
        scene.reset_counters()
        scene.frame_begin(6)
        if form == "plain":
            scene.launch(chunks)
        else:
            scene.launch_wavefront(chunks)
        c = scene.wait()
        assert c.errors == 0
        out[form] = scene.film() + (scene.counters(),)
    (ps, pc, pk), (ws, wc, wk) = out["plain"], out["wavefront"]
    assert np.array_equal(pc, wc)
    assert np.allclose(ps, ws, rtol=1e-12, atol=1e-12)
    for k in ("trace", "shadow_nee", "shadow_bsdf", "held", "samples", "errors", "stack_overflows"):
        assert pk[k] == wk[k], k
    scene.free()
