"""The work grid (x2_workgrid_*, host side) against the reference's own Grid (async_grid.h, compiled from source into
oracle/_ref) as the GPU lane uses it (every cell the GPU's), call by call: the same chunks in the same cells and order,
the same claims, frontiers, cellular choices and starting cells, under the progressive and flat orders, shares of a
frame, viewports and scores; the broker's launches against the reference feeder's claims restated over the reference
grid; and claims from many threads taking every chunk exactly once."""
import threading

import numpy as np
import pytest

import oracle_lib
from oracle_lib import RefWorkGrid, x2

needs_reference = pytest.mark.skipif(not oracle_lib.have_reference(), reason="oracle/_ref not built")
NONE = 0xFFFFFFFF

CASES = [
    # width, height, spp, options, viewport
    (256, 256, 64, {}, None),
    (1000, 700, 37, {"cell_size": 32, "samples_per_chunk": 5}, None),
    (517, 263, 16, {"progressive": 0, "samples_per_chunk": 3}, None),
    (640, 480, 9, {"samples_per_chunk": 2}, None),
    (384, 320, 64, {"sample_first": 16, "sample_count": 24}, None),
    (300, 200, 12, {"samples_per_chunk": 8}, (37, 21, 250, 170)),
    (64, 8, 5, {"cell_size": 8}, None),
]


def _make(case):
    width, height, spp, opts, view = case
    options = x2.workgrid_options(**opts)
    return x2.WorkGrid(width, height, spp, options, viewport=view), RefWorkGrid(width, height, spp, options, viewport=view)


@needs_reference
@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}x{c[1]}s{c[2]}-{i}" for i, c in enumerate(CASES)])
def test_grid_layout_matches_reference(case):
    mine, ref = _make(case)
    assert mine.cells == ref.cells
    assert mine.total == ref.total
    assert mine.ranges() == ref.ranges()
    assert mine.frontier() == ref.frontier()
    for i in range(mine.cells):
        assert mine.remaining(i) == ref.remaining(i)
        assert mine.claimable(i) == ref.claimable(i)
    # Each cell's claimable chunks in queue order (as far as the frontier lets one claim reach), then the rest.
    for sweep in range(3):
        for i in range(mine.cells):
            a = mine.claim(i, 1 << 20)
            b = ref.claim(i, 1 << 20)
            assert np.array_equal(a, b), (sweep, i)
            assert mine.frontier() == ref.frontier()


@needs_reference
@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}x{c[1]}s{c[2]}-{i}" for i, c in enumerate(CASES)])
def test_claims_and_choices_match_reference(case):
    """A seeded script of claims by the workers moving by the cellular rules, scores set part way (some unknown), then
    a drain: every answer of both grids equal."""
    mine, ref = _make(case)
    rng = np.random.default_rng(case[2] * 7 + case[0])
    cells = mine.cells
    workers = [mine.seed(w, 6) for w in range(6)]
    assert workers == [ref.seed(w, 6) for w in range(6)]
    steps = 0
    while steps < 4000:
        steps += 1
        if steps in (60, 400):
            scores = rng.random(cells).astype(np.float32)
            scores[rng.random(cells) < 0.2] = -1.0
            if steps == 400:
                scores[: cells // 2] = scores[0]  # ties: the hash decides
            mine.set_scores(scores)
            ref.set_scores(scores)
        w = int(rng.integers(0, len(workers)))
        cur = workers[w] if rng.random() < 0.9 else NONE
        a = mine.choose(cur, w)
        b = ref.choose(cur, w)
        assert a == b, f"step {steps}: choose({cur}, {w})"
        assert mine.frontier() == ref.frontier()
        if a == NONE:
            if mine.empty():
                assert ref.empty()
                break
            continue
        workers[w] = a
        n = int(rng.integers(1, 9))
        assert np.array_equal(mine.claim(a, n), ref.claim(a, n)), f"step {steps}: claim({a}, {n})"
    assert mine.empty() == ref.empty()
    for i in range(cells):
        assert mine.remaining(i) == ref.remaining(i)


@needs_reference
@pytest.mark.parametrize("want", [1, 7, 64, 1024, 1 << 20])
def test_broker_launches_match_reference_feeder(want):
    """The GPU broker's launches (x2_workgrid_take) against the reference feeder's claims over the reference grid, a
    GPU-only progressive frame drained launch by launch."""
    options = x2.workgrid_options(workers=32)
    mine = x2.WorkGrid(720, 480, 24, options)
    ref = RefWorkGrid(720, 480, 24, options)
    cells = [ref.seed(w, 32) for w in range(32)]
    launches = 0
    while True:
        a = mine.take(want)
        b = ref.take(want, cells)
        assert np.array_equal(a, b), f"launch {launches}"
        if not len(a):
            break
        launches += 1
    assert mine.empty() and ref.empty()
    assert launches >= 1


def test_progressive_ranges_and_frontier():
    g = x2.WorkGrid(128, 128, 20, x2.workgrid_options(samples_per_chunk=4))
    assert g.ranges() == [(0, 1), (1, 1), (2, 2), (4, 4), (8, 4), (12, 4), (16, 4)]
    flat = x2.WorkGrid(128, 128, 10, x2.workgrid_options(progressive=0, samples_per_chunk=4))
    assert flat.ranges() == [(0, 4), (4, 4), (8, 2)]
    share = x2.WorkGrid(128, 128, 64, x2.workgrid_options(sample_first=10, sample_count=7))
    assert share.ranges() == [(10, 1), (11, 1), (12, 2), (14, 3)]
    # The frontier holds each cell to the least range still unclaimed anywhere: cell 0 drains range 0 only.
    tiles = g.cell(0)["tiles"]
    assert tiles == 64
    got = g.claim(0, 1000)
    assert len(got) == tiles and set(got["first"]) == {0}
    assert g.frontier() == 0
    for i in range(1, g.cells):
        g.claim(i, 1000)
    assert g.frontier() == 1
    # A closed grid hands out nothing.
    g.close()
    assert g.empty() and len(g.claim(0, 10)) == 0


def test_claims_from_many_threads_take_each_chunk_once():
    g = x2.WorkGrid(512, 512, 32, x2.workgrid_options(progressive=0, samples_per_chunk=2))
    total = g.total
    taken = [[] for _ in range(8)]

    def worker(k):
        rng = np.random.default_rng(k)
        while not g.empty():
            cell = int(rng.integers(0, g.cells))
            c = g.claim(cell, int(rng.integers(1, 17)))
            if len(c):
                taken[k].append(c)

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(8)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    allc = np.concatenate([c for t in taken for c in t])
    assert len(allc) == total
    keys = allc["tile"].astype(np.int64) * 1000 + allc["first"]
    assert len(np.unique(keys)) == total


def test_bad_grids_are_refused():
    with pytest.raises(x2.X2Error):
        x2.WorkGrid(0, 10, 4)
    with pytest.raises(x2.X2Error):
        x2.WorkGrid(64, 64, 4, x2.workgrid_options(cell_size=12))
    with pytest.raises(x2.X2Error):
        x2.WorkGrid(64, 64, 4, x2.workgrid_options(samples_per_chunk=0))


@needs_reference
def test_appended_passes_match_reference():
    """An adaptive frame's grid: cells start empty and the coordinator appends each pass's chunks; the workers' claims
    against the reference's grid fed the same appends, every answer equal."""
    options = x2.workgrid_options(cell_size=32)
    mine = x2.WorkGrid(300, 200, 16, options, empty=True)
    ref = RefWorkGrid(300, 200, 16, options, empty=True)
    assert mine.total == ref.total == 0 and mine.ranges() == ref.ranges() == []
    rng = np.random.default_rng(11)
    tiles_x = (300 + 7) // 8
    cells_x = (300 + 31) // 32
    for p in range(6):
        for cell in range(mine.cells):
            cx, cy = cell % cells_x, cell // cells_x
            tiles = [ty * tiles_x + tx for ty in range(cy * 4, min(25, cy * 4 + 4)) for tx in range(cx * 4, min(tiles_x, cx * 4 + 4))]
            keep = [t for t in tiles if rng.random() < 0.6]
            chunks = np.zeros(len(keep), x2.CHUNK_DTYPE)
            chunks["tile"], chunks["first"], chunks["count"], chunks["cell"] = keep, p << 16, 4, cell
            mine.append(cell, chunks)
            ref.append(cell, chunks)
        assert mine.total == ref.total
        for _ in range(200):
            cur = int(rng.integers(0, mine.cells))
            a, b = mine.choose(cur, 3), ref.choose(cur, 3)
            assert a == b
            if a == NONE:
                break
            n = int(rng.integers(1, 12))
            assert np.array_equal(mine.claim(a, n), ref.claim(a, n))
        for i in range(mine.cells):
            assert mine.remaining(i) == ref.remaining(i)


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_ranks_shares_cover_the_frame_once(world):
    """Each rank's grid is its share of the frame (x2.lanes.share: sample_first, sample_count): drained, the ranks'
    chunks together cover every tile's samples [0, spp) exactly once, in the progressive order within each share."""
    from x2 import lanes

    width, height, spp = 200, 136, 37
    tiles = ((width + 7) // 8) * ((height + 7) // 8)
    cover = np.zeros((tiles, spp), np.int32)
    for rank in range(world):
        first, count = lanes.share(rank, world, spp)
        g = x2.WorkGrid(width, height, spp, x2.workgrid_options(sample_first=first, sample_count=count))
        while True:
            c = g.take(1000)
            if not len(c):
                break
            for t, f, n in zip(c["tile"], c["first"], c["count"]):
                cover[t, f:f + n] += 1
        assert g.empty()
    assert (cover == 1).all()
