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


@pytest.fixture(scope="module")
def ragged(ctx):
    """The closed box at 250 x 190: partial tiles on the right and bottom edges, regions clamped to the image."""
    s = x2.SyntheticScene(0)
    cfg = x2.Config.from_buffer_copy(s.config)
    cfg.width, cfg.height = 250, 190
    s.config = cfg
    return s, x2.Scene(ctx, s.desc, cfg)


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


def _replay(scene, cfg, target, min_samples, max_samples, cellular, budget=0):
    """Renders an adaptive frame and replays the reference's frame on the host against it: the reference's schedule,
    and before each pass past the uniform ones its pixelError of the film so far and its region trees' masks (cellular:
    its next generation, a live tile sampling all its pixels); each active pixel then takes the pass's next samples.
    Each pass's film is rebuilt from the samples' own radiance (the per-sample API), summed as the device sums it (each
    pixel's samples of the pass in order, then added to the pixel), so the replay's plan and film equal the device's
    bit for bit."""
    if budget:
        result = scene.render_adaptive_budget(min_samples, max_samples, target, budget)
    else:
        result = scene.render_adaptive(min_samples, max_samples, target, cellular=cellular)
    planned = scene.adaptive_planned().astype(np.int64)
    sums, odd, counts = scene.film(odd=True)
    pixels = cfg.width * cfg.height
    offsets = np.concatenate([[0], np.cumsum(planned)[:-1]])
    pix = np.repeat(np.arange(pixels), planned).astype(np.uint32)
    idx = (np.arange(int(planned.sum())) - np.repeat(offsets, planned)).astype(np.uint32)
    rgba, status = scene.integrate(pix, idx)
    assert (status == x2.DONE).all()
    assert np.array_equal(rgba, rgba.astype(np.float32).astype(np.float64))
    tiles_x, tiles_y = (cfg.width + 7) // 8, (cfg.height + 7) // 8
    tile_of = (np.arange(pixels) // cfg.width // 8) * tiles_x + (np.arange(pixels) % cfg.width) // 8
    in_image = np.zeros(tiles_x * tiles_y, np.uint64)
    for t in range(len(in_image)):
        x0, y0 = (t % tiles_x) * 8, (t // tiles_x) * 8
        m = 0
        for b in range(64):
            if x0 + b % 8 < cfg.width and y0 + b // 8 < cfg.height:
                m |= 1 << b
        in_image[t] = m
    cells = oracle_lib.RefCellular(cfg.width, cfg.height, target, in_image) if cellular else None
    film = np.zeros((pixels, 4))
    film_odd = np.zeros((pixels, 4))
    film_counts = np.zeros(pixels, np.uint32)
    plan = np.zeros(pixels, np.int64)
    converged, passes, generations, spent = False, 0, [], 0
    for k, (start, end) in enumerate(oracle_lib.reference_adaptive_schedule(max_samples)):
        size = end - start
        if start < min_samples:
            active = np.arange(pixels)
        else:
            if budget and spent >= budget:
                break
            errors = oracle_lib.reference_pixel_errors(film, film_odd, film_counts)
            if cellular:
                left = max(0, budget - spent)
                live = cells.update_budget(errors, plan, left, max_samples, target) if budget else cells.update(errors)
                if live == 0:
                    converged = True
                    break
                alive = cells.alive()
                generations.append(live)
                if budget:
                    # The reference's pass under a budget (async_render.h:1376-1395): the live tiles furthest above the
                    # target first, while each fits in what is left.
                    ratio = cells.ratio()
                    cost = np.array([bin(int(m)).count("1") for m in in_image]) * size
                    live_tiles = [t for t in range(len(in_image)) if in_image[t] and alive[t]]
                    if sum(cost[t] for t in live_tiles) > left:
                        kept, taken = np.zeros_like(alive), 0
                        for t in sorted(live_tiles, key=lambda t: -ratio[t]):
                            if taken + cost[t] > left:
                                break
                            taken += cost[t]
                            kept[t] = 1
                        alive = kept
                active = np.nonzero(alive[tile_of])[0]
            else:
                masks, done = oracle_lib.reference_adaptive_masks(cfg.width, cfg.height, target, errors)
                if done:
                    converged = True
                    break
                tiles = np.nonzero(masks)[0]
                bits = ((masks[tiles, None] >> np.arange(64, dtype=np.uint64)) & np.uint64(1)).astype(bool)
                t, b = np.nonzero(bits)
                x = (tiles[t] % tiles_x) * 8 + b % 8
                y = (tiles[t] // tiles_x) * 8 + b // 8
                active = np.sort(y * cfg.width + x)
            if len(active) == 0:
                converged = True
                break
        assert (plan[active] + size <= planned[active]).all(), f"the replay wants more samples than the device planned at pass {k}"
        first = offsets[active] + plan[active]
        block = rgba[first[:, None] + np.arange(size)]  # active x size x 4, in sample order
        film[active] += np.cumsum(block, axis=1)[:, -1]
        is_odd = ((plan[active, None] + np.arange(size)) & 1).astype(bool)
        film_odd[active] += np.cumsum(np.where(is_odd[:, :, None], block, 0.0), axis=1)[:, -1]
        film_counts[active] += size
        plan[active] += size
        spent += len(active) * size
        passes += 1
    print(result, "replay: passes", passes, "converged", converged, "live tiles a generation", generations)
    assert np.array_equal(plan, planned), f"{int(np.count_nonzero(plan != planned))} pixels planned differently"
    assert result["passes"] == passes and bool(result["converged"]) == converged
    assert np.array_equal(counts, film_counts)
    assert np.array_equal(sums, film), f"max abs diff {np.abs(sums - film).max()}"
    assert np.array_equal(odd, film_odd), f"max abs diff {np.abs(odd - film_odd).max()}"
    return result, generations


@needs_reference
def test_adaptive_frame_replays_reference_frame(box):
    s, scene = box
    _replay(scene, s.config, 0.0005, 4, 256, cellular=False)


@needs_reference
@pytest.mark.parametrize("target", [0.002, 0.0005])
def test_cellular_frame_replays_reference_frame(box, target):
    """The cellular generations' frame against the reference's Cellular replayed on the host, bit for bit; the
    generations thin out as tiles converge."""
    s, scene = box
    result, generations = _replay(scene, s.config, target, 4, 256, cellular=True)
    assert len(generations) >= 2 and min(generations) < max(generations)


@needs_reference
@pytest.mark.parametrize("budget", [3_000_000, 9_000_000])
def test_budget_frame_replays_reference_frame(box, budget):
    """A frame by sampling generations under a budget of samples against the reference's Cellular with its Budget
    (and the pass's tile choice under the budget) replayed on the host, bit for bit; it spends about its budget."""
    s, scene = box
    result, generations = _replay(scene, s.config, 0.0, 4, 256, cellular=True, budget=budget)
    assert result["samples"] <= budget + s.config.width * s.config.height * 32
    assert result["samples"] >= 0.5 * budget


@needs_reference
@pytest.mark.parametrize("cellular", [False, True])
def test_ragged_frame_replays_reference_frame(ragged, cellular):
    """Trees and cellular generations on an image whose edge tiles are partial, against the reference replayed."""
    s, scene = ragged
    _replay(scene, s.config, 0.001, 4, 128, cellular=cellular)



def test_adaptive_arguments_refused(box):
    s, scene = box
    for call in (lambda: scene.render_adaptive(4, 0, 0.001), lambda: scene.render_adaptive(4, 64, 0.0),
                 lambda: scene.render_adaptive(4, 64, -1.0, cellular=True), lambda: scene.render_adaptive_budget(4, 64, 0.0, 0),
                 lambda: scene.render_adaptive_budget(4, 64, -1.0, 1000)):
        with pytest.raises(x2.X2Error) as e:
            call()
        assert e.value.code == x2.EINVAL
