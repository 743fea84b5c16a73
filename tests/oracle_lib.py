"""Loaders for the oracle (test infrastructure only): the plain-C sampler restatement (oracle/liboracle_sampler.so)
and the reference integrator compiled from the reference's own sources (oracle/_ref/libx2ref.so).
"""
import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "xpu2-foundation_b200"))
import x2  # noqa: E402

SAMPLER = os.path.join(ROOT, "oracle", "liboracle_sampler.so")
REFERENCE = os.path.join(ROOT, "oracle", "_ref", "libx2ref.so")
REPLAY = os.path.join(ROOT, "oracle", "_ref", "libx2ref_replay.so")  # oracle/replay.h


def sampler():
    lib = C.CDLL(SAMPLER)
    u32, u64, vp = C.c_uint32, C.c_uint64, C.c_void_p
    lib.oracle_sampling_words.argtypes = [vp, vp, u64, u32, vp]
    lib.oracle_philox.argtypes = [vp, vp, u64, vp]
    lib.oracle_sobol.argtypes = [u32, u32]
    lib.oracle_sobol.restype = u32
    lib.oracle_direction.argtypes = [u32, u32]
    lib.oracle_direction.restype = u32
    lib.oracle_child_branch.argtypes = [u64, u32, u32]
    lib.oracle_child_branch.restype = u64
    lib.oracle_unit.argtypes = [u32]
    lib.oracle_unit.restype = C.c_float
    lib.oracle_word.argtypes = [u32, u64, u64, u64, u32]
    lib.oracle_word.restype = u32
    return lib


def sampling_words(lib, ids, dims, policy):
    ids = np.ascontiguousarray(ids, dtype=x2.IDENTITY_DTYPE)
    dims = np.ascontiguousarray(dims, dtype=np.uint32)
    out = np.empty(len(dims), np.uint32)
    lib.oracle_sampling_words(ids.ctypes.data, dims.ctypes.data, len(dims), policy, out.ctypes.data)
    return out


# x2_diag_call (include/x2_diag.h) and the replay build's backend event (oracle/replay.h).
CALL_DTYPE = np.dtype([("fn", np.uint32), ("a", np.float32), ("b", np.float32), ("r0", np.float32), ("r1", np.float32)])
EVENT_DTYPE = np.dtype([("kind", np.uint32), ("value", np.uint32), ("t", np.float32), ("x", np.float32), ("y", np.float32),
                        ("z", np.float32)])


def have_reference():
    return os.path.exists(REFERENCE)


_generator = None


def generator():
    """The reference build's copy of the seeded scene generator (x2_scene_generate, compiled into libx2ref.so), for
    processes that must not load libx2 (the timed reference arm)."""
    global _generator
    if _generator is None:
        lib = C.CDLL(REFERENCE)
        lib.x2_scene_generate.argtypes = [C.c_uint32, C.c_uint64, C.POINTER(C.POINTER(x2.SceneDesc)), C.POINTER(x2.Config)]
        lib.x2_scene_generate.restype = C.c_int
        lib.x2_scene_desc_free.argtypes = [C.POINTER(x2.SceneDesc)]
        lib.x2_scene_desc_free.restype = None
        _generator = lib
    return _generator


class Reference:
    """The reference's integratePaths (async_integrator.h:1986) over a scene, on host threads."""

    def __init__(self, synthetic, config=None, path=REFERENCE):
        self.lib = lib = C.CDLL(path)
        vp, u32, u64, i32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int
        lib.x2ref_open.argtypes = [C.POINTER(x2.SceneDesc), C.POINTER(x2.Config)]
        lib.x2ref_open.restype = vp
        lib.x2ref_close.argtypes = [vp]
        lib.x2ref_integrate.argtypes = [vp, vp, u64, vp, vp, i32]
        lib.x2ref_integrate.restype = i32
        lib.x2ref_render.argtypes = [vp, u32, u32, i32, vp, vp, vp, vp]
        lib.x2ref_render.restype = i32
        lib.x2ref_render_tiles.argtypes = [vp, vp, u32, u32, u32, i32, vp, vp]
        lib.x2ref_render_tiles.restype = i32
        lib.x2ref_trace.argtypes = [vp, vp, u64, vp, vp, vp]
        lib.x2ref_trace.restype = i32
        lib.x2ref_sample_words.argtypes = [vp, vp, u64, u32, vp]
        lib.x2ref_sample_words.restype = i32
        lib.x2ref_child_branch.argtypes = [u64, u32, u32]
        lib.x2ref_child_branch.restype = u64
        cfg = synthetic.config if config is None else config
        self.config = cfg
        self._desc_counts = (synthetic.desc.material_count, synthetic.desc.light_count)
        self.h = lib.x2ref_open(synthetic.desc_ptr, C.byref(cfg))
        if not self.h:
            raise RuntimeError("x2ref_open failed")

    def close(self):
        if self.h:
            self.lib.x2ref_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def integrate(self, pixels, indices, threads=None):
        pairs = np.ascontiguousarray(np.stack([np.asarray(pixels, np.uint32), np.asarray(indices, np.uint32)], 1))
        n = len(pairs)
        rgba = np.empty((n, 4), np.float64)
        status = np.empty(n, np.uint32)
        rc = self.lib.x2ref_integrate(self.h, pairs.ctypes.data, n, rgba.ctypes.data, status.ctypes.data, threads or os.cpu_count())
        assert rc == 0
        return rgba, status

    def render(self, first, count, threads=None):
        p = self.config.width * self.config.height
        sums = np.zeros((p, 4))
        odd = np.zeros((p, 4))
        counts = np.zeros(p, np.uint32)
        rays = np.zeros(4, np.uint64)
        rc = self.lib.x2ref_render(self.h, first, count, threads or os.cpu_count(), sums.ctypes.data, odd.ctypes.data, counts.ctypes.data,
                                   rays.ctypes.data)
        return rc, sums, odd, counts, rays

    def render_tiles(self, tiles, first, count, threads=None):
        """A bounded sample of a frame: the given tiles' pixels x samples [first, first+count). Returns (rc,
        samples rendered, ray counts [trace, nee, bsdf, held])."""
        tiles = np.ascontiguousarray(tiles, np.uint32)
        samples = np.zeros(1, np.uint64)
        rays = np.zeros(4, np.uint64)
        rc = self.lib.x2ref_render_tiles(self.h, tiles.ctypes.data, len(tiles), first, count, threads or os.cpu_count(), samples.ctypes.data,
                                         rays.ctypes.data)
        return rc, int(samples[0]), rays

    def render_tiles_film(self, tiles, first, count, threads=None):
        """The given tiles' film: (rc, sums [tiles, 64, 4] FP64, counts [tiles, 64]); tile k's position pos is pixel
        tilePixel(tiles[k], pos) (row-major 8x8 within the tile)."""
        tiles = np.ascontiguousarray(tiles, np.uint32)
        sums = np.zeros((len(tiles), 64, 4))
        counts = np.zeros((len(tiles), 64), np.uint32)
        f = self.lib.x2ref_render_tiles_film
        f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, C.c_void_p, C.c_void_p]
        f.restype = C.c_int
        rc = f(self.h, tiles.ctypes.data, len(tiles), first, count, threads or os.cpu_count(), sums.ctypes.data, counts.ctypes.data)
        return rc, sums, counts

    def replay(self, pixel, index, table=None):
        """One sample through the replay build (Reference(..., path=REPLAY); oracle/replay.h) with the given
        transcendental values (records as x2_diag_call, or None: libm's own). Returns (rgba, status, calls made, backend
        events, table misses)."""
        cap = 1 << 16
        calls = np.zeros(cap, CALL_DTYPE)
        events = np.zeros(cap, EVENT_DTYPE)
        rgba = np.zeros(4)
        status, nc, ne, misses = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint64()
        table = np.ascontiguousarray(table if table is not None else np.zeros(0, CALL_DTYPE), CALL_DTYPE)
        f = self.lib.x2ref_replay
        f.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                      C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
        f.restype = C.c_int
        rc = f(self.h, int(pixel), int(index), table.ctypes.data, len(table), rgba.ctypes.data, C.byref(status), calls.ctypes.data, cap,
               C.byref(nc), events.ctypes.data, cap, C.byref(ne), C.byref(misses))
        assert rc == 0
        return rgba, status.value, calls[: min(cap, nc.value)], events[: min(cap, ne.value)], misses.value

    def trace(self, rays, brute=False):
        """Closest hit (triangle, t) and occlusion through the oracle's BVH, or by testing every triangle."""
        rays = np.ascontiguousarray(rays, np.float32)
        n = len(rays)
        tri = np.empty(n, np.uint32)
        t = np.empty(n, np.float32)
        occ = np.empty(n, np.uint32)
        f = self.lib.x2ref_trace_brute if brute else self.lib.x2ref_trace
        f.argtypes = [C.c_void_p] * 2 + [C.c_uint64] + [C.c_void_p] * 3
        f(self.h, rays.ctypes.data, n, tri.ctypes.data, t.ctypes.data, occ.ctypes.data)
        return tri, t, occ


def reference_sampling_words(ids, dims, policy):
    lib = C.CDLL(REFERENCE)
    lib.x2ref_sample_words.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_uint32, C.c_void_p]
    ids = np.ascontiguousarray(ids, dtype=x2.IDENTITY_DTYPE)
    dims = np.ascontiguousarray(dims, dtype=np.uint32)
    out = np.empty(len(dims), np.uint32)
    lib.x2ref_sample_words(ids.ctypes.data, dims.ctypes.data, len(dims), policy, out.ctypes.data)
    return out


def random_identities(n, seed):
    """Seeded identities exercising every field: 32-bit pixels, 64-bit indices (high bits too), streams, branches."""
    r = np.random.default_rng(seed)
    ids = np.zeros(n, x2.IDENTITY_DTYPE)
    ids["pixel"] = r.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    idx = r.integers(0, 2**63, n, dtype=np.uint64)
    small = r.random(n) < 0.5
    idx[small] = r.integers(0, 4096, small.sum(), dtype=np.uint64)
    ids["index"] = idx
    ids["stream"] = r.integers(0, 2**63, n, dtype=np.uint64)
    ids["branch"] = r.integers(0, 2**63, n, dtype=np.uint64)
    return ids


def sample_pairs(config, n, seed):
    """n seeded (pixel, index) samples of a frame."""
    r = np.random.default_rng(seed)
    pixels = r.integers(0, config.width * config.height, n).astype(np.uint32)
    indices = r.integers(0, config.spp, n).astype(np.uint32)
    return pixels, indices


def adjoint64(ref, first, count, dldi, threads=None, params=None, masses=False, texels=0, texture=None):
    """The FP64 CPU adjoint (oracle/adjoint64.h) of samples [first, first + count) of every pixel, given dL/dimage
    (pixels x 3): (albedo grads [materials, 3], roughness grads [materials], radiance grads [lights, 3], image sums
    [pixels, 3]), all FP64, and with `masses` the gradients' credit masses (sums of credit magnitudes) in the same
    shapes. `params` = (albedo, roughness, radiance) arrays (None entries kept) set first; `texture` (an array) sets
    texture 0's texels first; with `texels` > 0 the texel gradients (texels x 3) come last."""
    lib = ref.lib
    vp = C.c_void_p
    lib.x2ref_adjoint64.argtypes = [vp, C.c_uint32, C.c_uint32, vp, C.c_int, vp, vp, vp, vp, vp, vp]
    if texture is not None:
        t = np.ascontiguousarray(texture, np.float32)
        lib.x2ref_set_texture.argtypes = [vp, C.c_uint32, vp]
        assert lib.x2ref_set_texture(ref.h, 0, t.ctypes.data) == 0
    lib.x2ref_adjoint64.restype = C.c_int
    lib.x2ref_set_params.argtypes = [vp, vp, vp, vp]
    lib.x2ref_set_params.restype = C.c_int
    if params is not None:
        arrs = [None if a is None else np.ascontiguousarray(a, np.float32) for a in params]
        ptrs = [None if a is None else a.ctypes.data for a in arrs]
        assert lib.x2ref_set_params(ref.h, *ptrs) == 0
    d = ref._desc_counts
    dldi = np.ascontiguousarray(dldi, np.float32)
    ga = np.zeros((d[0], 3))
    gg = np.zeros(d[0])
    gr = np.zeros((d[1], 3))
    img = np.zeros((ref.config.width * ref.config.height, 3))
    mass = np.zeros(4 * d[0] + 3 * d[1])
    tg = np.zeros((texels, 3)) if texels else None
    rc = lib.x2ref_adjoint64(ref.h, first, count, dldi.ctypes.data, threads or os.cpu_count(), ga.ctypes.data, gg.ctypes.data,
                             gr.ctypes.data, img.ctypes.data, mass.ctypes.data, tg.ctypes.data if texels else None)
    assert rc == 0, rc
    out = (ga, gg, gr, img)
    if masses:
        M = d[0]
        out = out + ((mass[:3 * M].reshape(M, 3), mass[3 * M:4 * M], mass[4 * M:].reshape(-1, 3)),)
    if texels:
        out = out + (tg,)
    return out


def reference_pixel_errors(sums, odd, counts):
    """The reference's pixelError (async_integrator.h:3109) of every pixel of a film."""
    lib = C.CDLL(REFERENCE)
    lib.x2ref_pixel_errors.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]
    sums = np.ascontiguousarray(sums, np.float64)
    odd = np.ascontiguousarray(odd, np.float64)
    counts = np.ascontiguousarray(counts, np.uint32)
    out = np.empty(len(counts), np.float32)
    lib.x2ref_pixel_errors(sums.ctypes.data, odd.ctypes.data, counts.ctypes.data, len(counts), out.ctypes.data)
    return out


class RefCellular:
    """The reference's cellular generations (async_adaptive.h Cellular) over a width x height image's tiles."""

    def __init__(self, width, height, target, in_image):
        lib = self.lib = C.CDLL(REFERENCE)
        lib.x2ref_cellular_open.argtypes = [C.c_int, C.c_int, C.c_float, C.c_void_p, C.c_uint32]
        lib.x2ref_cellular_open.restype = C.c_void_p
        lib.x2ref_cellular_free.argtypes = [C.c_void_p]
        lib.x2ref_cellular_update.argtypes = [C.c_void_p, C.c_void_p]
        lib.x2ref_cellular_update.restype = C.c_uint64
        lib.x2ref_cellular_alive.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
        in_image = np.ascontiguousarray(in_image, np.uint64)
        self.tiles = len(in_image)
        self._h = lib.x2ref_cellular_open(width, height, target, in_image.ctypes.data, self.tiles)

    def update(self, errors):
        """The next generation from per-pixel errors; its live tiles' count."""
        errors = np.ascontiguousarray(errors, np.float32)
        return int(self.lib.x2ref_cellular_update(self._h, errors.ctypes.data))

    def update_budget(self, errors, planned, remaining, most, floor):
        """The next generation under a budget (Budget: each pixel's planned samples, the samples left, the most a pixel
        may have, the error floor); its live tiles' count."""
        f = self.lib.x2ref_cellular_update_budget
        f.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_double, C.c_uint32, C.c_float]
        f.restype = C.c_uint64
        errors = np.ascontiguousarray(errors, np.float32)
        planned = np.ascontiguousarray(planned, np.uint32)
        return int(f(self._h, errors.ctypes.data, planned.ctypes.data, len(planned), remaining, most, floor))

    def ratio(self):
        f = self.lib.x2ref_cellular_ratio
        f.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
        out = np.zeros(self.tiles, np.float32)
        f(self._h, out.ctypes.data, self.tiles)
        return out

    def alive(self):
        out = np.zeros(self.tiles, np.uint8)
        self.lib.x2ref_cellular_alive(self._h, out.ctypes.data, self.tiles)
        return out

    def __del__(self):
        try:
            self.lib.x2ref_cellular_free(self._h)
        except Exception:
            pass


def reference_adaptive_schedule(max_samples):
    """The reference's pass schedule (async_adaptive.h schedule): [(start, end)] sample ranges a pixel."""
    lib = C.CDLL(REFERENCE)
    lib.x2ref_adaptive_schedule.argtypes = [C.c_uint32, C.c_void_p, C.c_uint32]
    lib.x2ref_adaptive_schedule.restype = C.c_uint32
    out = np.zeros(2 * 1024, np.uint32)
    n = lib.x2ref_adaptive_schedule(max_samples, out.ctypes.data, 1024)
    return [(int(out[2 * k]), int(out[2 * k + 1])) for k in range(min(n, 1024))]


def reference_adaptive_masks(width, height, target, errors):
    """The reference's region trees (async_adaptive.h Regions) over per-pixel errors: (tile masks, all converged)."""
    lib = C.CDLL(REFERENCE)
    lib.x2ref_adaptive_masks.argtypes = [C.c_uint32, C.c_uint32, C.c_float, C.c_void_p, C.c_void_p, C.c_void_p]
    errors = np.ascontiguousarray(errors, np.float32)
    masks = np.empty(((width + 7) // 8) * ((height + 7) // 8), np.uint64)
    done = np.zeros(1, np.uint32)
    lib.x2ref_adaptive_masks(width, height, target, errors.ctypes.data, masks.ctypes.data, done.ctypes.data)
    return masks, bool(done[0])


class RefWorkGrid:
    """The reference's own work grid (async_grid.h Grid, compiled from source into oracle/_ref) as the GPU lane uses it
    (GridOptions::mode 1: every cell the GPU's; every claim and choice the GPU's), call by call, with the same methods
    as x2.WorkGrid."""

    GPU = 1  # Device::Gpu, and GridOptions::mode for a GPU-only grid

    def __init__(self, width, height, spp, options, empty=False, viewport=None):
        lib = self.lib = C.CDLL(REFERENCE)
        vp, u32, u64 = C.c_void_p, C.c_uint32, C.c_uint64
        sig = {
            "x2ref_grid_open": ([u32, u32, u32, u32, u32, C.c_int, C.c_int, u32, u32, vp, u32, C.c_int, vp], vp),
            "x2ref_grid_free": ([vp], None), "x2ref_grid_cells": ([vp], u32), "x2ref_grid_total": ([vp], u64),
            "x2ref_grid_ranges": ([vp, vp, u32], u32),
            "x2ref_grid_claim": ([vp, u32, u32, vp, u32], u32), "x2ref_grid_claimable": ([vp, u32, u32], u32),
            "x2ref_grid_remaining": ([vp, u32], u32), "x2ref_grid_empty": ([vp], u32), "x2ref_grid_frontier": ([vp, u32], u32),
            "x2ref_grid_choose": ([vp, u32, u32, u32], u32), "x2ref_grid_seed": ([vp, u32, u32, u32], u32),
            "x2ref_grid_set_scores": ([vp, vp, u32], None), "x2ref_grid_append": ([vp, u32, vp, u32], None),
            "x2ref_grid_close": ([vp], None),
        }
        for name, (args, res) in sig.items():
            f = getattr(lib, name)
            f.argtypes = args
            f.restype = res
        view = None if viewport is None else np.ascontiguousarray(viewport, np.int32)
        self._view = view
        self._h = lib.x2ref_grid_open(width, height, spp, options.cell_size, options.samples_per_chunk, self.GPU, options.progressive,
                                      options.sample_first, options.sample_count, None, 0, int(bool(empty)),
                                      None if view is None else view.ctypes.data)
        assert self._h, "the reference grid refused its arguments"

    def free(self):
        if self._h:
            self.lib.x2ref_grid_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    @property
    def cells(self):
        return self.lib.x2ref_grid_cells(self._h)

    @property
    def total(self):
        return self.lib.x2ref_grid_total(self._h)

    def ranges(self):
        out = np.zeros(2 * 4096, np.uint32)
        n = self.lib.x2ref_grid_ranges(self._h, out.ctypes.data, 4096)
        return [(int(out[2 * k]), int(out[2 * k + 1])) for k in range(n)]

    def claim(self, cell, n):
        out = np.zeros(max(n, 1), x2.CHUNK_DTYPE)
        got = self.lib.x2ref_grid_claim(self._h, cell, n, out.ctypes.data, self.GPU)
        return out[:got]

    def claimable(self, cell):
        return self.lib.x2ref_grid_claimable(self._h, cell, self.GPU)

    def remaining(self, cell):
        return self.lib.x2ref_grid_remaining(self._h, cell)

    def empty(self):
        return bool(self.lib.x2ref_grid_empty(self._h))

    def frontier(self):
        return self.lib.x2ref_grid_frontier(self._h, self.GPU)

    def choose(self, current, salt):
        return self.lib.x2ref_grid_choose(self._h, self.GPU, current, salt)

    def seed(self, worker, workers):
        return self.lib.x2ref_grid_seed(self._h, self.GPU, worker, workers)

    def set_scores(self, scores):
        scores = np.ascontiguousarray(scores, np.float32)
        self.lib.x2ref_grid_set_scores(self._h, scores.ctypes.data, len(scores))

    def append(self, cell, chunks):
        chunks = np.ascontiguousarray(chunks, dtype=x2.CHUNK_DTYPE)
        self.lib.x2ref_grid_append(self._h, cell, chunks.ctypes.data, len(chunks))

    def close(self):
        self.lib.x2ref_grid_close(self._h)

    def take(self, want, cells):
        """The reference feeder's claims for one GPU launch (async_render.h:784-797), restated over this grid: `cells`
        (the GPU's cellular workers' cells, seeded by the caller with seed()) move as the feeder moves them."""
        out, got = [], 0
        share = (want + len(cells) - 1) // len(cells)
        for w in range(len(cells)):
            if got >= want:
                break
            need, moves = min(share, want - got), 0
            while need and moves < 8:
                cell = self.choose(cells[w], w)
                if cell == 0xFFFFFFFF:
                    break
                cells[w] = cell
                c = self.claim(cell, need)
                out.append(c)
                got += len(c)
                need -= len(c)
                moves += 1
        return np.concatenate(out) if out else np.zeros(0, x2.CHUNK_DTYPE)


