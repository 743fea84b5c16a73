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
    grid = x2.WorkGrid(cfg.width, cfg.height, spp, x2.workgrid_options(mode=x2.WORKGRID_GPU, samples_per_chunk=4))
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
    grid = x2.WorkGrid(cfg.width, cfg.height, 64, x2.workgrid_options(mode=x2.WORKGRID_GPU, sample_first=8, sample_count=8))
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
