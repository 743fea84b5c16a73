"""Frames fed from the work grid by the GPU broker (x2_render_workgrid): the progressive order's launches render the
same samples as a uniform frame — every pixel's counts exact, the audit clean, the sums those of the uniform frame up
to the order of their FP64 additions — and a share of a frame holds exactly its sample range."""
import numpy as np
import pytest

from oracle_lib import x2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def box(ctx):
    s = x2.SyntheticScene(0)
    return s, x2.Scene(ctx, s.desc, s.config)


def _uniform(scene, first, count):
    scene.frame_begin(count)
    scene.render_frame_wavefront(first, count)
    scene.wait()
    return scene.film()


@pytest.mark.parametrize("per_launch", [97, 1024, 1 << 20])
def test_progressive_frame_equals_uniform_frame(box, per_launch):
    s, scene = box
    cfg = s.config
    spp = 24
    grid = x2.WorkGrid(cfg.width, cfg.height, spp, x2.workgrid_options(samples_per_chunk=4))
    r = scene.render_workgrid(grid, per_launch)
    sums, counts = scene.film()
    print(per_launch, r)
    pixels = cfg.width * cfg.height
    assert r["samples"] == pixels * spp and r["chunks"] == grid.total
    assert r["launches"] == (1 if per_launch >= grid.total else -(-grid.total // per_launch))
    assert grid.empty()
    assert (counts == spp).all()
    scene.audit(np.full(pixels, spp, np.uint32))
    usums, ucounts = _uniform(scene, 0, spp)
    assert np.array_equal(counts, ucounts)
    assert np.allclose(sums, usums, rtol=1e-12, atol=1e-15)


def test_share_of_a_frame(box):
    s, scene = box
    cfg = s.config
    grid = x2.WorkGrid(cfg.width, cfg.height, 64, x2.workgrid_options(sample_first=8, sample_count=8))
    r = scene.render_workgrid(grid, 4096)
    sums, counts = scene.film()
    assert (counts == 8).all() and r["samples"] == cfg.width * cfg.height * 8
    usums, _ = _uniform(scene, 8, 8)
    assert np.allclose(sums, usums, rtol=1e-12, atol=1e-15)


def test_mismatched_grid_is_refused(box):
    s, scene = box
    grid = x2.WorkGrid(s.config.width + 8, s.config.height, 4)
    with pytest.raises(x2.X2Error):
        scene.render_workgrid(grid, 64)


def _cell_scores(sums, counts, width, height, cell):
    """The reference's cellScores (async_render.h:1581-1611) over the preview picture of HostFilm::preview
    (async_cpu.h:1359-1379: each pixel's sum over its count, as float32), restated in numpy with float32 tones and the
    cells' FP64 sums taken in the reference's pixel order."""
    n = counts.astype(np.float64)
    rgb = np.where(counts[:, None] > 0, (sums[:, :3] / np.maximum(n, 1)[:, None]).astype(np.float32), np.float32(0))
    lum = (np.float32(0.2126) * rgb[:, 0] + np.float32(0.7152) * rgb[:, 1]) + np.float32(0.0722) * rgb[:, 2]
    with np.errstate(invalid="ignore", over="ignore"):
        tone = np.where(np.isfinite(lum) & (lum > 0), lum / (np.float32(1) + lum), np.float32(0)).astype(np.float32)
    covered = (counts > 0).reshape(height, width)
    tone = tone.reshape(height, width)
    d = np.zeros((height, width), np.float64)
    left = np.zeros_like(covered)
    left[:, 1:] = covered[:, :-1]
    up = np.zeros_like(covered)
    up[1:, :] = covered[:-1, :]
    dl = np.zeros((height, width), np.float32)
    dl[:, 1:] = np.abs(tone[:, 1:] - tone[:, :-1])
    du = np.zeros((height, width), np.float32)
    du[1:, :] = np.abs(tone[1:, :] - tone[:-1, :])
    d = np.where(left, dl.astype(np.float64), 0.0)
    d = d + np.where(up, du.astype(np.float64), 0.0)
    cx, cy = (width + cell - 1) // cell, (height + cell - 1) // cell
    scores = np.full(cx * cy, -1.0, np.float32)
    for c in range(cx * cy):
        x0, y0 = (c % cx) * cell, (c // cx) * cell
        block = d[y0:y0 + cell, x0:x0 + cell][covered[y0:y0 + cell, x0:x0 + cell]]
        if len(block):
            scores[c] = np.float32(np.cumsum(block)[-1] / len(block))
    return scores


def test_cell_scores_from_the_film(box):
    """Important parts first: the cells' scores computed on the device from a film where a third of the tiles have
    samples equal the reference's cellScores restated over the same film, bit for bit."""
    s, scene = box
    cfg = s.config
    tiles = ((cfg.width + 7) // 8) * ((cfg.height + 7) // 8)
    sel = np.arange(0, tiles, 3, dtype=np.uint32)
    chunks = np.zeros(len(sel), x2.CHUNK_DTYPE)
    chunks["tile"], chunks["first"], chunks["count"] = sel, 0, 4
    scene.frame_begin(4)
    scene.launch_wavefront(chunks)
    scene.wait()
    sums, counts = scene.film()
    grid = x2.WorkGrid(cfg.width, cfg.height, 16, x2.workgrid_options(cell_size=32))
    got = scene.score_workgrid(grid)
    want = _cell_scores(sums, counts, cfg.width, cfg.height, 32)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), f"{int(np.count_nonzero(got != want))} cells differ"
    assert (got > 0).sum() > 0
