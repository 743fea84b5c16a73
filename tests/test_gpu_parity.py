"""GPU parity tests (B200): the CUDA path through the C ABI against the oracle — the reference's own sampler and
integrator — on the same seeded inputs.

Bars: random words bit-exact; per-pixel sample counts exact; triangle choices exact; per-sample radiance within
RTOL = 1e-4 relative (FP32 reassociation and the device's sincosf against libm's), with a floor of ATOL = 1e-6 for
values near zero.
"""
import os

import numpy as np
import pytest

import oracle_lib
from oracle_lib import x2

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RTOL, ATOL = 1e-4, 1e-6
needs_reference = pytest.mark.skipif(not oracle_lib.have_reference(), reason="oracle/_ref not built")


def within(a, b):
    return np.abs(a - b) <= RTOL * np.abs(b) + ATOL


# ---- sampler ----
@pytest.mark.parametrize("policy", [0, 3, 15])
def test_sampler_golden(ctx, policy):
    g = np.load(os.path.join(GOLDEN, "sampler_words.npz"))
    assert np.array_equal(ctx.sample_words(g["ids"], g["dims"], policy), g[f"p{policy}"])


def test_sampler_16m_words(ctx):
    """16,777,216 words, device against the C restatement, as the reference's run_sample_core.py compares them."""
    sam = oracle_lib.sampler()
    n = 1 << 24
    ids = oracle_lib.random_identities(n, seed=2024)
    dims = np.random.default_rng(3).integers(0, 1100, n).astype(np.uint32)
    for policy in (15, 0):
        dev = ctx.sample_words(ids, dims, policy)
        assert np.array_equal(dev, oracle_lib.sampling_words(sam, ids, dims, policy))


def test_sampler_config0_identities(ctx):
    """Every camera and first-bounce dimension of config 0's identities (65,536 px x 16 spp) under policy 15."""
    sam = oracle_lib.sampler()
    px = np.repeat(np.arange(256 * 256, dtype=np.uint32), 16)
    idx = np.tile(np.arange(16, dtype=np.uint64), 256 * 256)
    ids = np.zeros(len(px), x2.IDENTITY_DTYPE)
    ids["pixel"], ids["index"], ids["stream"] = px, idx, 1
    for d in (0, 1, 16, 17, 18, 19, 20, 300):
        dims = np.full(len(px), d, np.uint32)
        assert np.array_equal(ctx.sample_words(ids, dims, 15), oracle_lib.sampling_words(sam, ids, dims, 15)), d


# ---- scenes ----
@pytest.fixture(scope="module")
def box(ctx):
    s = x2.SyntheticScene(0)
    return s, x2.Scene(ctx, s.desc, s.config)


@pytest.fixture(scope="module")
def field(ctx):
    s = x2.SyntheticScene(108)
    return s, x2.Scene(ctx, s.desc, s.config)


@pytest.fixture(scope="module")
def textured(ctx):
    """Config 44: the differentiable scene shrunk, its heightfield's diffuse colour a 64x64 texture read at the
    vertices' uvs (UsdUVTexture: bilinear on primary paths, the closest texel on indirect ones)."""
    s = x2.SyntheticScene(44)
    return s, x2.Scene(ctx, s.desc, s.config)


def _scene(cid, box, field, textured):
    return box if cid == 0 else field if cid == 108 else textured


# ---- traversal ----
def random_rays(scene_desc, n, seed, shadow=False):
    r = np.random.default_rng(seed)
    v = np.ctypeslib.as_array(scene_desc.vertices, (scene_desc.vertex_count, 3))
    lo, hi = v.min(0), v.max(0)
    o = lo + (hi - lo) * r.random((n, 3))
    d = r.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    near = np.zeros(n)
    far = np.full(n, 3.4e38) if not shadow else r.random(n) * np.linalg.norm(hi - lo)
    return np.concatenate([o, d, near[:, None], far[:, None]], 1).astype(np.float32)


@needs_reference
@pytest.mark.parametrize("which", ["box", "field"])
def test_traversal_matches_oracle(which, box, field):
    """Closest-hit triangle and t, and any-hit occlusion, exactly as the oracle's traversal finds them."""
    s, scene = box if which == "box" else field
    rays = np.concatenate([random_rays(s.desc, 100000, 1), random_rays(s.desc, 100000, 2, shadow=True)])
    tri, t, occ = scene.trace_rays(rays)
    ref = oracle_lib.Reference(s)
    rtri, rt, rocc = ref.trace(rays)
    bad = np.flatnonzero((tri != rtri) | (occ != rocc))
    if len(bad):
        btri, bt, bocc = ref.trace(rays[bad[:50]], brute=True)
        rows = [f"ray {i} {rays[i].tolist()}: device ({tri[i]}, {t[i]!r}, {occ[i]}) oracle ({rtri[i]}, {rt[i]!r}, {rocc[i]}) "
                f"brute ({b}, {bb!r}, {o})" for i, b, bb, o in zip(bad[:5], btri, bt, bocc)]
        pytest.fail(f"{len(bad)} of {len(rays)} rays differ:\n" + "\n".join(rows))
    assert np.array_equal(t[tri != 0xFFFFFFFF], rt[rtri != 0xFFFFFFFF])
    assert scene.counters()["stack_overflows"] == 0


@needs_reference
def test_oracle_traversal_matches_brute_force(box):
    """The oracle's own BVH against testing every triangle (the box scene's 34)."""
    s, _ = box
    rays = np.concatenate([random_rays(s.desc, 20000, 3), random_rays(s.desc, 20000, 4, shadow=True)])
    ref = oracle_lib.Reference(s)
    a = ref.trace(rays)
    b = ref.trace(rays, brute=True)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


# ---- per-sample radiance ----
@pytest.mark.parametrize("cid", [0, 108, 44])
def test_radiance_golden(cid, box, field, textured):
    g = np.load(os.path.join(GOLDEN, f"radiance_c{cid}.npz"))
    s, scene = _scene(cid, box, field, textured)
    rgba, status = scene.integrate(g["pixels"], g["indices"])
    assert np.array_equal(status, g["status"])
    ok = within(rgba, g["rgba"]).all(axis=1)
    bad = np.flatnonzero(~ok)
    assert ok.all(), f"{len(bad)} of {len(ok)} samples outside {RTOL}: first {bad[:8]}: {rgba[bad[:3]]} vs {g['rgba'][bad[:3]]}"


# The samples of the live test outside the per-sample bar, by configuration: config 108's two are each a one-ulp
# difference of CUDA's sincosf against the host libm's sincos on a sampled angle, amplified continuously with no
# discrete decision flipped (tests/test_gpu_parity_cause.py: they vanish with the functions rounded from double, and
# the reference replayed with the device's function values gives the device's radiance bit for bit).
EXPECTED_OUTSIDE = {0: set(), 108: {(22444, 55), (26184, 27)}, 44: set()}


@needs_reference
@pytest.mark.parametrize("cid", [0, 108, 44])
def test_radiance_live_reference(cid, box, field, textured):
    """Many more samples against the live reference build: every sample within tolerance except the listed, explained
    ones (EXPECTED_OUTSIDE); every status and every alpha must agree."""
    s, scene = _scene(cid, box, field, textured)
    px, idx = oracle_lib.sample_pairs(s.config, 60000, 1000 + cid)
    rgba, status = scene.integrate(px, idx)
    ref = oracle_lib.Reference(s)
    rrgba, rstatus = ref.integrate(px, idx)
    assert np.array_equal(status, rstatus)
    assert np.array_equal(rgba[:, 3], rrgba[:, 3])
    ok = within(rgba, rrgba).all(axis=1)
    rel = (np.abs(rgba - rrgba) / np.maximum(np.abs(rrgba), 1e-6)).max(axis=1)
    print(f"config {cid}: {ok.mean() * 100:.4f}% of {len(ok)} samples within {RTOL}; outside: {np.sort(rel[~ok])[::-1][:8]}")
    outside = {(int(p), int(i)) for p, i in zip(px[~ok], idx[~ok])}
    assert outside == EXPECTED_OUTSIDE[cid], f"samples outside {RTOL}: {sorted(outside)}"


# ---- film and audit ----
@needs_reference
def test_film_and_audit_box(box):
    s, scene = box
    scene.frame_begin(16)
    scene.render_frame(0, 16)
    c = scene.wait()
    assert c.errors == 0
    scene.audit()
    sums, counts = scene.film()
    assert (counts == 16).all()
    ref = oracle_lib.Reference(s)
    rc, rsums, _, rcounts, rays = ref.render(0, 16)
    assert rc == 0 and np.array_equal(counts, rcounts)
    # per pixel: sums of 16 samples each within the per-sample bar (plus rounding of the sum order)
    close = np.abs(sums - rsums) <= 16 * (RTOL * np.abs(rsums) / 16 + ATOL)
    assert close.all(axis=1).mean() >= 0.999
    cnt = scene.counters()
    assert cnt["errors"] == 0 and cnt["stack_overflows"] == 0


def test_film_equals_sum_of_samples(field):
    """The film of a frame is the sum of its samples' radiance (the lane's film against the per-sample API)."""
    s, scene = field
    cfg = s.config
    scene.frame_begin(3)
    scene.render_frame(5, 3)
    scene.wait()
    sums, counts = scene.film()
    assert (counts == 3).all()
    p = cfg.width * cfg.height
    px = np.repeat(np.arange(p, dtype=np.uint32), 3)
    idx = np.tile(np.arange(5, 8, dtype=np.uint32), p)
    rgba, status = scene.integrate(px, idx)
    assert (status == x2.DONE).all()
    want = rgba.reshape(p, 3, 4).sum(1)
    assert np.allclose(sums, want, rtol=1e-12, atol=1e-12)


def test_audit_catches_missing_samples(box):
    s, scene = box
    scene.frame_begin(16)
    tiles = (256 // 8) * (256 // 8)
    chunks = np.zeros(tiles, x2.CHUNK_DTYPE)
    chunks["tile"] = np.arange(tiles)
    chunks["first"] = 0
    chunks["count"] = 16
    chunks["count"][37] = 15  # one tile short of a sample
    scene.launch(chunks)
    scene.wait()
    with pytest.raises(x2.X2Error) as e:
        scene.audit()
    assert e.value.code == x2.EAUDIT
    assert "pixel" in str(e.value)


def test_chunked_launches_ragged_image(ctx):
    """An image whose edge tiles are partial, rendered by uneven chunks over two launches in flight."""
    s = x2.SyntheticScene(108)
    cfg = s.config
    cfg.width, cfg.height, cfg.spp = 250, 130, 5
    scene = x2.Scene(ctx, s.desc, cfg)
    scene.frame_begin(4)
    tiles = ((250 + 7) // 8) * ((130 + 7) // 8)
    a = np.zeros(tiles, x2.CHUNK_DTYPE)
    a["tile"], a["first"], a["count"] = np.arange(tiles), 0, 4
    b = np.zeros(tiles, x2.CHUNK_DTYPE)
    b["tile"], b["first"], b["count"] = np.arange(tiles), 4, 1
    scene.launch(a)
    scene.launch(b)
    c = scene.wait()
    assert c.samples == 250 * 130 * 5 and c.errors == 0
    scene.audit()


def test_rejects_bad_input(box, ctx):
    s, scene = box
    scene.frame_begin(4)
    bad = np.zeros(1, x2.CHUNK_DTYPE)
    bad["tile"] = 10**6
    bad["count"] = 1
    with pytest.raises(x2.X2Error) as e:
        scene.launch(bad)
    assert e.value.code == x2.EINVAL
    bad["tile"], bad["count"] = 0, 5  # more samples than the frame's chunks hold
    with pytest.raises(x2.X2Error):
        scene.launch(bad)
    rgba, status = scene.integrate(np.array([256 * 256], np.uint32), np.array([0], np.uint32))  # pixel out of range
    assert status[0] == x2.ERROR
    empty = scene.integrate(np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    assert len(empty[1]) == 0
