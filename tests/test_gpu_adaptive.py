"""Adaptive sampling (the reference's adaptive frame: pixelError, MoonRay's region trees, the GPU pass chain): the
device chain's errors and tile masks against the reference's own pixelError and Regions (compiled from source) on the
same films, bit for bit; and whole adaptive frames — their sample counts audited against the chain's plan, each pixel
holding exactly its planned samples [0, n)."""
import numpy as np
import pytest

import oracle_lib
from oracle_lib import x2

pytestmark = pytest.mark.gpu
needs_reference = pytest.mark.skipif(not oracle_lib.have_reference(), reason="oracle/_ref not built")


@pytest.fixture(scope="module")
def box(ctx):
    s = x2.SyntheticScene(0)
    return s, x2.Scene(ctx, s.desc, s.config)


@needs_reference
@pytest.mark.parametrize("spp,target", [(5, 0.05), (16, 0.02), (16, 0.002), (37, 0.01)])
def test_chain_matches_reference_trees(box, spp, target):
    s, scene = box
    cfg = s.config
    scene.frame_begin_adaptive(spp)
    scene.render_frame_wavefront(0, spp)
    scene.wait()
    sums, odd, counts = scene.film(odd=True)
    errors, masks, stop = scene.adaptive_step(target, 0, 4)
    want = oracle_lib.reference_pixel_errors(sums, odd, counts)
    assert np.array_equal(errors.view(np.uint32), want.view(np.uint32)), "pixel errors differ from the reference's"
    ref_masks, done = oracle_lib.reference_adaptive_masks(cfg.width, cfg.height, target, want)
    active = int(np.count_nonzero(ref_masks))
    print(f"spp {spp} target {target}: {active} of {len(ref_masks)} tiles active, converged {done}")
    assert bool(stop) == done
    if not done:
        assert np.array_equal(masks, ref_masks), f"{int(np.count_nonzero(masks != ref_masks))} tile masks differ"


def test_adaptive_frame(box):
    s, scene = box
    cfg = s.config
    result = scene.render_adaptive(4, 256, 0.0005)
    planned = scene.adaptive_planned()
    sums, odd, counts = scene.film(odd=True)
    print(result, "samples a pixel: min", planned.min(), "max", planned.max(), "mean", planned.mean())
    assert result["samples"] == int(planned.sum())
    assert np.array_equal(counts, planned)
    scene.audit(planned)
    assert planned.min() >= 4 and planned.max() <= 256
    assert planned.max() > planned.min()  # samples went where the error was
    # Each pixel holds exactly its samples [0, n): its sums equal those samples' radiance added up.
    rng = np.random.default_rng(3)
    pix = rng.choice(cfg.width * cfg.height, 64, replace=False)
    px = np.repeat(pix, planned[pix]).astype(np.uint32)
    idx = np.concatenate([np.arange(n) for n in planned[pix]]).astype(np.uint32)
    rgba, status = scene.integrate(px, idx)
    assert (status == x2.DONE).all()
    owner = np.repeat(np.arange(len(pix)), planned[pix])
    want = np.zeros((len(pix), 4))
    np.add.at(want, owner, rgba)
    assert np.allclose(sums[pix], want, rtol=1e-9, atol=1e-12)
    odd_want = np.zeros((len(pix), 4))
    sel = (idx & 1) == 1
    np.add.at(odd_want, owner[sel], rgba[sel])
    assert np.allclose(odd[pix], odd_want, rtol=1e-9, atol=1e-12)
