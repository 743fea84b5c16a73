"""CPU tests: the oracle pinned against the reference's own known answers and the reference compiled from source;
the scene generator; the C ABI library loads and exports every declared symbol (no device calls)."""
import ctypes as C
import json
import os
import re

import numpy as np
import pytest

import oracle_lib
from oracle_lib import x2

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def sam():
    return oracle_lib.sampler()


def test_philox_known_answers(sam):
    """The three Philox4x32-10 vectors of the reference's sample_fixture.h:17-20."""
    kat = json.load(open(os.path.join(GOLDEN, "philox_kat.json")))
    for v in kat["philox"]:
        c = np.array(v["counter"], np.uint32)
        k = np.array(v["key"], np.uint32)
        out = np.empty(4, np.uint32)
        sam.oracle_philox(c.ctypes.data, k.ctypes.data, 1, out.ctypes.data)
        assert out.tolist() == v["out"]


def test_word_known_answer(sam):
    """word(Identity{5,3,1,0}, 0) = 0xf05db22f, as the reference's sampler prints it."""
    kat = json.load(open(os.path.join(GOLDEN, "philox_kat.json")))
    assert sam.oracle_word(5, 3, 1, 0, 0) == kat["word_5_3_1_0_dim0"]


def test_sobol_first_points(sam):
    """qmc_fixture.h:14-15: the first eight Sobol points of dimensions 0..3, in units of 2^-3."""
    kat = json.load(open(os.path.join(GOLDEN, "philox_kat.json")))
    for d in range(4):
        assert [sam.oracle_sobol(i, d) >> 29 for i in range(8)] == kat["sobol_first8"][d]


def test_unit_bounds(sam):
    """sample_fixture.h:50: unit(0) = 0, unit(~0) = 1 - 2^-24 < 1."""
    assert sam.oracle_unit(0) == 0.0
    assert sam.oracle_unit(0xFFFFFFFF) == np.float32(1.0 - 2.0**-24)


@pytest.mark.parametrize("policy", [0, 3, 15])
def test_sampling_words_golden(sam, policy):
    """The restatement against samplingWord of the reference compiled from source (golden vectors)."""
    g = np.load(os.path.join(GOLDEN, "sampler_words.npz"))
    got = oracle_lib.sampling_words(sam, g["ids"], g["dims"], policy)
    assert np.array_equal(got, g[f"p{policy}"])


@pytest.mark.skipif(not oracle_lib.have_reference(), reason="oracle/_ref not built")
def test_sampling_words_live_reference(sam):
    """200k fresh identities x dimensions x policies against the reference's own samplingWord."""
    ids = oracle_lib.random_identities(50000, seed=99)
    r = np.random.default_rng(5)
    dims = r.integers(0, 64, len(ids)).astype(np.uint32)
    for policy in (0, 1, 2, 4, 8, 15):
        assert np.array_equal(oracle_lib.sampling_words(sam, ids, dims, policy), oracle_lib.reference_sampling_words(ids, dims, policy))


def test_stratification(sam):
    """qmc_fixture.h:17-21: every power-of-two prefix fills each 1-D stratum once after the scramble."""
    for pixel in range(4):
        for d in (0, 1, 16, 17):
            n = 1024
            ids = np.zeros(n, x2.IDENTITY_DTYPE)
            ids["pixel"] = pixel
            ids["index"] = np.arange(n)
            ids["stream"] = 19
            ids["branch"] = 3
            w = oracle_lib.sampling_words(sam, ids, np.full(n, d, np.uint32), 3)
            for m in range(1, 11):
                cells = w[: 1 << m] >> (32 - m)
                assert len(np.unique(cells)) == 1 << m


def test_elementary_intervals(sam):
    """qmc_fixture.h:26-30: the camera's 2-D net has one point in every elementary rectangle."""
    n = 256
    ids = np.zeros(n, x2.IDENTITY_DTYPE)
    ids["pixel"] = 19
    ids["index"] = np.arange(n)
    ids["stream"] = 713
    a = oracle_lib.sampling_words(sam, ids, np.zeros(n, np.uint32), 3)
    b = oracle_lib.sampling_words(sam, ids, np.ones(n, np.uint32), 3)
    for k in range(9):
        ca = (a >> (32 - k)) if k else np.zeros(n, np.uint32)
        cb = (b >> (24 + k)) if k < 8 else np.zeros(n, np.uint32)
        cell = (ca.astype(np.uint64) << (8 - k)) | cb
        assert len(np.unique(cell)) == n


@pytest.mark.skipif(not oracle_lib.have_reference(), reason="oracle/_ref not built")
def test_child_branch_matches_reference(sam):
    lib = C.CDLL(oracle_lib.REFERENCE)
    lib.x2ref_child_branch.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32]
    lib.x2ref_child_branch.restype = C.c_uint64
    r = np.random.default_rng(1)
    for _ in range(1000):
        p, a, b = int(r.integers(0, 2**63)), int(r.integers(0, 2**16)), int(r.integers(0, 2**16))
        assert sam.oracle_child_branch(p, a, b) == lib.x2ref_child_branch(p, a, b)


def test_scene_generator_deterministic():
    a, b = x2.SyntheticScene(108), x2.SyntheticScene(108)
    for k, v in a.arrays().items():
        assert np.array_equal(v, b.arrays()[k]), k
    assert a.desc.triangle_count == 8 * 8 * 512 + 31 * 5120
    c0 = x2.SyntheticScene(0)
    assert c0.desc.triangle_count == 10 + 24 and c0.config.spp == 16 and c0.config.width == 256


def test_config1_triangle_count():
    """Config 1 as specified: 64x64 tiles of 16x16 quads + 2000 level-4 icospheres = 12,337,152 triangles."""
    s = x2.SyntheticScene(1)
    assert s.desc.triangle_count == 64 * 64 * 16 * 16 * 2 + 2000 * 20 * 4**4 == 12337152
    assert s.config.width == 1920 and s.config.height == 1080 and s.config.spp == 64 and s.config.max_depth == 12
    assert s.desc.light_count == 17


@pytest.mark.skipif(not oracle_lib.have_reference(), reason="oracle/_ref not built")
@pytest.mark.parametrize("cid", [0, 108, 33])
def test_oracle_radiance_golden(cid):
    """The live reference build reproduces the committed golden radiance bit for bit (same build flags)."""
    g = np.load(os.path.join(GOLDEN, f"radiance_c{cid}.npz"))
    s = x2.SyntheticScene(cid)
    ref = oracle_lib.Reference(s)
    rgba, status = ref.integrate(g["pixels"], g["indices"])
    assert np.array_equal(status, g["status"])
    assert np.array_equal(rgba, g["rgba"])


def test_library_exports_every_declared_symbol():
    """libx2.so loads (no device needed) and exports every function include/x2.h declares."""
    header = open(os.path.join(oracle_lib.ROOT, "include", "x2.h")).read()
    names = set(re.findall(r"\b(x2_[a-z0-9_]+)\s*\(", header))
    assert len(names) >= 25
    lib = x2.library()
    for n in sorted(names):
        assert hasattr(lib, n), n
    assert lib.x2_version().startswith(b"x2-b200")


def test_diagnostic_library_exports_its_switches():
    """libx2diag.so (the diagnostic build) loads and exports every function include/x2.h and include/x2_diag.h
    declare; the product library exports none of x2_diag.h's."""
    import ctypes

    names = set()
    for h in ("x2.h", "x2_diag.h"):
        names |= set(re.findall(r"\b(x2_[a-z0-9_]+)\s*\(", open(os.path.join(oracle_lib.ROOT, "include", h)).read()))
    diag = ctypes.CDLL(x2.DIAG_LIBRARY)
    for n in sorted(names):
        assert hasattr(diag, n), n
    assert not hasattr(x2.library(), "x2_diag_set")


@pytest.fixture(scope="module")
def adjoint_scene():
    if not oracle_lib.have_reference():
        pytest.skip("oracle/_ref not built")
    s = x2.SyntheticScene(44)
    ref = oracle_lib.Reference(s)
    yield s, ref
    ref.close()


def test_fp64_adjoint_primal_matches_reference(adjoint_scene):
    """The FP64 CPU adjoint's own primal (oracle/adjoint64.h, the estimator restated in double) against the reference
    integrator compiled from source on the same samples: pixel sums within 1e-4 relative on almost every pixel (a
    shadow ray that grazes an edge can go the other way once its direction is computed in double), and the image
    mean within 2e-4 (near-mirror GGX lobes' values, which the reference computes in float, move it most)."""
    s, ref = adjoint_scene
    cfg = s.config
    w = np.zeros((cfg.width * cfg.height, 3), np.float32)
    _, _, _, img = oracle_lib.adjoint64(ref, 0, cfg.spp, w + 1.0)
    rc, sums, _, counts, _ = ref.render(0, cfg.spp)
    assert rc == 0 and (counts == cfg.spp).all()
    want = sums[:, :3]
    ok = (np.abs(img - want) <= 1e-4 * np.abs(want) + 1e-6).all(1)
    assert ok.mean() >= 0.97
    assert abs(img.mean() - want.mean()) <= 2e-4 * want.mean()


def test_fp64_adjoint_against_finite_differences(adjoint_scene):
    """The FP64 adjoint's albedo and radiance gradients against central differences of its own FP64 primal with
    common random numbers. Both parameters enter linearly; the differences also see Russian roulette's decisions
    flip (their noise grows as 1 / step and falls with the samples), so the check takes 128 samples a pixel and a 5%
    step: within 1% of the gradient plus 0.2% of the largest of its kind."""
    s, ref = adjoint_scene
    cfg = s.config
    d = s.desc
    spp = 128
    albedo = np.array([list(d.materials[m].diffuse) for m in range(d.material_count)], np.float64)
    radiance = np.array([list(d.lights[i].radiance) for i in range(d.light_count)], np.float64)
    kinds = np.array([d.materials[m].kind for m in range(d.material_count)])
    w = np.random.default_rng(11).random((cfg.width * cfg.height, 3)).astype(np.float32)
    ga, gg, gr, _ = oracle_lib.adjoint64(ref, 0, spp, w, params=(albedo, None, radiance))
    assert np.all(ga[kinds != x2.MAT_LAMBERT] == 0) and np.all(gg[kinds != x2.MAT_GGX] == 0)

    def loss(a, r):
        _, _, _, img = oracle_lib.adjoint64(ref, 0, spp, w, params=(a, None, r))
        return float((img / spp * w).sum())

    lam = np.flatnonzero(kinds == x2.MAT_LAMBERT)
    for m in lam[np.argsort(-np.abs(ga[lam, 1]))][:3]:
        h = 5e-2 * albedo[m, 1]
        up, down = albedo.copy(), albedo.copy()
        up[m, 1] += h
        down[m, 1] -= h
        fd = (loss(up, radiance) - loss(down, radiance)) / (2 * h)
        assert abs(fd - ga[m, 1]) <= 1e-2 * abs(ga[m, 1]) + 2e-3 * np.abs(ga[:, 1]).max(), (m, fd, ga[m, 1])
    for i in np.argsort(-np.abs(gr[:, 0]))[:3]:
        h = 5e-2 * radiance[i, 0]
        up, down = radiance.copy(), radiance.copy()
        up[i, 0] += h
        down[i, 0] -= h
        fd = (loss(albedo, up) - loss(albedo, down)) / (2 * h)
        assert abs(fd - gr[i, 0]) <= 1e-2 * abs(gr[i, 0]) + 2e-3 * np.abs(gr[:, 0]).max(), (i, fd, gr[i, 0])
    oracle_lib.adjoint64(ref, 0, cfg.spp, w, params=(albedo, None, radiance))


@pytest.mark.skipif(not oracle_lib.have_reference(), reason="oracle/_ref not built")
def test_oracle_traversal_matches_brute_force_on_a_field():
    """The oracle's own BVH against testing every triangle on config 108 (the 1M-triangle field scaled down: 191,488
    triangles): 10,000 closest-hit rays and 10,000 shadow rays of random origins and directions inside the scene's
    bounds, the same triangle, t and occlusion. The device traversal is checked against this BVH, so a defect shared by
    both would have to survive this check too."""
    r = np.random.default_rng(108)
    s = x2.SyntheticScene(108)
    v = np.ctypeslib.as_array(s.desc.vertices, (s.desc.vertex_count, 3))
    lo, hi = v.min(0), v.max(0)
    rays = []
    for shadow in (False, True):
        o = lo + (hi - lo) * r.random((10000, 3))
        d = r.normal(size=(10000, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        far = r.random(10000) * np.linalg.norm(hi - lo) if shadow else np.full(10000, 3.4e38)
        rays.append(np.concatenate([o, d, np.zeros((10000, 1)), far[:, None]], 1).astype(np.float32))
    rays = np.concatenate(rays)
    ref = oracle_lib.Reference(s)
    a = ref.trace(rays)
    b = ref.trace(rays, brute=True)
    hits = int((a[0] != 0xFFFFFFFF).sum())
    assert hits > 5000, hits  # most rays hit something: the check is not vacuous
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
