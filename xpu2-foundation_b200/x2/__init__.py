"""x2 — Python layer over the B200 path-sample engine's C ABI (libx2.so, include/x2.h).

Mirrors the reference's two interfaces for the path: the per-sample `integrate(config, pixel, index, backend, out)`
(xpu2/interactive/async_integrator.h:3047) as `Scene.integrate`, and the GPU lane
(xpu2/interactive/async_gpu.h:1372-1707: begin / launch / poll / downloadFilm / sums / counts) as
`Scene.frame_begin / launch / poll / wait / film / audit`. Errors raise `X2Error` with the library's message, as
the reference's `cpu::need` raises `std::runtime_error`.

There is no CPU fallback: without the built library or a CUDA device every call raises.
"""
import ctypes as C
import os
import weakref

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# X2_LIBRARY may name the diagnostic build (libx2diag.so: the product's kernels plus the x2_diag_* switches of
# include/x2_diag.h) for a parity investigation; the product is libx2.so.
LIBRARY = os.environ.get("X2_LIBRARY") or os.path.join(_HERE, "libx2.so")
DIAG_LIBRARY = os.path.join(_HERE, "libx2diag.so")

OK, EINVAL, ECUDA, ENOMEM, ETIMEOUT, EAUDIT, ENODEV, EDEVICE = range(8)
DONE, MISS, ERROR, SKIP, DEFER = range(5)
MAT_LAMBERT, MAT_GGX = 0, 1
LIGHT_ENV, LIGHT_RECT = 0, 1


class X2Error(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"x2 error {code}: {message}")
        self.code = code


class Identity(C.Structure):
    _fields_ = [("pixel", C.c_uint32), ("pad", C.c_uint32), ("index", C.c_uint64), ("stream", C.c_uint64), ("branch", C.c_uint64)]


class Chunk(C.Structure):
    _fields_ = [("tile", C.c_uint32), ("first", C.c_uint32), ("count", C.c_uint32), ("cell", C.c_uint32)]


class Material(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("diffuse", C.c_float * 3), ("specular", C.c_float * 3), ("emission", C.c_float * 3),
                ("roughness", C.c_float), ("diffuse_texture", C.c_uint32)]


class Texture(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("wrap", C.c_uint32), ("pad", C.c_uint32), ("rgb", C.POINTER(C.c_float))]


class Light(C.Structure):
    _fields_ = [("type", C.c_uint32), ("sidedness", C.c_uint32), ("visible_in_camera", C.c_uint32), ("hemispherical", C.c_uint32),
                ("radiance", C.c_float * 3), ("position", C.c_float * 3), ("direction", C.c_float * 3),
                ("local2render", (C.c_float * 3) * 3), ("render2local", (C.c_float * 3) * 3), ("render2local_rot", (C.c_float * 3) * 3),
                ("scale", C.c_float), ("inv_area", C.c_float), ("plane_offset", C.c_float), ("half_width", C.c_float),
                ("half_height", C.c_float), ("visibility_mask", C.c_uint32), ("cos_theta_max", C.c_float),
                ("versine_theta_max", C.c_float)]


class Volume(C.Structure):
    _fields_ = [("bound_lo", C.c_float * 3), ("bound_hi", C.c_float * 3), ("density_grid", C.c_uint32), ("emission_grid", C.c_uint32),
                ("interpolation", C.c_uint32), ("feature_size", C.c_float), ("world_to_grid", C.c_float * 12), ("gain", C.c_float * 3),
                ("color_mult", C.c_float * 3), ("incandescence", C.c_float * 3), ("g", C.c_float), ("light_set", C.c_uint32),
                ("surface_opacity_threshold", C.c_float)]


class Grid(C.Structure):
    _fields_ = [("channels", C.c_uint32), ("lo", C.c_int32 * 3), ("dims", C.c_int32 * 3), ("world_to_index", C.c_double * 16),
                ("values", C.POINTER(C.c_float))]


class Camera(C.Structure):
    _fields_ = [("raster_to_camera", (C.c_float * 4) * 4), ("camera_to_render", (C.c_float * 4) * 4), ("near_clip", C.c_float),
                ("far_clip", C.c_float)]


class SceneDesc(C.Structure):
    _fields_ = [("vertex_count", C.c_uint32), ("triangle_count", C.c_uint32), ("mesh_count", C.c_uint32), ("material_count", C.c_uint32),
                ("light_count", C.c_uint32), ("pad", C.c_uint32), ("vertices", C.POINTER(C.c_float)), ("triangles", C.POINTER(C.c_uint32)),
                ("mesh_first", C.POINTER(C.c_uint32)), ("mesh_material", C.POINTER(C.c_uint32)), ("materials", C.POINTER(Material)),
                ("lights", C.POINTER(Light)), ("camera", Camera), ("volume_count", C.c_uint32), ("grid_count", C.c_uint32),
                ("volumes", C.POINTER(Volume)), ("grids", C.POINTER(Grid)), ("texture_count", C.c_uint32), ("pad2", C.c_uint32),
                ("textures", C.POINTER(Texture)), ("uvs", C.POINTER(C.c_float))]


_U = C.c_uint32
_F = C.c_float


class Config(C.Structure):
    """mixed::Config's fields this engine reads (gpu_jobs.h:10-44), with its defaults (x2_config_defaults)."""
    _fields_ = [("width", _U), ("height", _U), ("seed", _U), ("spp", _U), ("sampling", _U), ("filter", _U), ("filter_width", _F),
                ("light_count", _U), ("bsdf_samples", _U), ("light_samples", _U), ("max_depth", _U), ("max_diffuse_depth", _U),
                ("clamp_depth", _U), ("rr_threshold", _F), ("clamp_value", _F), ("max_glossy_depth", _U), ("max_mirror_depth", _U),
                ("max_hair_depth", _U), ("max_presence_depth", _U), ("shadow_terminator_fix", _U), ("roughness_clamping", _F),
                ("transparency_threshold", _F), ("visible_lights", _U), ("presence_threshold", _F), ("presence_quality", _F),
                ("shadow_reuse", _U), ("volume_count", _U), ("max_volume_depth", _U), ("volume_illumination_samples", _U),
                ("volume_overlap_mode", _U), ("volume_transmittance_threshold", _F), ("volume_attenuation_factor", _F),
                ("volume_contribution_factor", _F), ("volume_phase_attenuation_factor", _F), ("inv_volume_quality", _F),
                ("inv_volume_shadow_quality", _F), ("volume_estimator", _U), ("reserved", _U * 7)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class Counters(C.Structure):
    _fields_ = [("trace", C.c_uint64), ("shadow_nee", C.c_uint64), ("shadow_bsdf", C.c_uint64), ("held", C.c_uint64),
                ("samples", C.c_uint64), ("errors", C.c_uint64), ("stack_overflows", C.c_uint64), ("pad", C.c_uint64)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_ if k != "pad"}


class Request(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("first", C.c_uint32), ("count", C.c_uint32)]


class WavefrontShape(C.Structure):
    FIELDS = ("paths", "refill", "blocks_per_sm", "trace_blocks", "shade_blocks", "tri_limit", "batch_window", "lobe_queues",
              "shadow_order", "extend_bins", "short_stack", "shade_split", "light_split", "tri_overlap")
    _fields_ = [(f, C.c_uint32) for f in FIELDS]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k in self.FIELDS}


def wavefront_shape_defaults():
    s = WavefrontShape()
    library().x2_wavefront_shape_defaults(C.byref(s))
    return s


class AdaptiveResult(C.Structure):
    _fields_ = [("passes", C.c_uint32), ("converged", C.c_uint32), ("samples", C.c_uint64), ("milliseconds", C.c_float), ("pad", C.c_uint32)]


class WorkGridOptions(C.Structure):
    _fields_ = [("cell_size", C.c_uint32), ("samples_per_chunk", C.c_uint32), ("progressive", C.c_uint32),
                ("sample_first", C.c_uint32), ("sample_count", C.c_uint32), ("workers", C.c_uint32)]


class WorkGridResult(C.Structure):
    _fields_ = [("launches", C.c_uint64), ("chunks", C.c_uint64), ("samples", C.c_uint64), ("milliseconds", C.c_float),
                ("gpu_milliseconds", C.c_float)]


class Completion(C.Structure):
    _fields_ = [("launch", C.c_uint64), ("samples", C.c_uint64), ("errors", C.c_uint64), ("milliseconds", C.c_float), ("pad", C.c_uint32)]


_lib = None


def library():
    """The loaded libx2.so (ctypes), its signatures declared. Raises when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBRARY):
        raise X2Error(ENODEV, f"{LIBRARY} is not built (run xpu2-foundation_b200/build.py)")
    lib = C.CDLL(LIBRARY)
    vp, u32, u64, i32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int
    sig = {
        "x2_version": ([], C.c_char_p), "x2_last_error": ([], C.c_char_p), "x2_config_defaults": ([C.POINTER(Config)], None),
        "x2_open": ([i32, C.POINTER(vp)], i32), "x2_close": ([vp], i32), "x2_synchronize": ([vp, i32], i32),
        "x2_sample_words": ([vp, vp, vp, u64, u32, vp], i32), "x2_sample_words_device": ([vp, vp, vp, u64, u32, vp], i32),
        "x2_scene_load": ([vp, C.POINTER(SceneDesc), C.POINTER(vp)], i32), "x2_scene_free": ([vp], i32),
        "x2_config_set": ([vp, C.POINTER(Config)], i32),
        "x2_scene_info": ([vp, C.POINTER(u64), C.POINTER(u64), C.POINTER(u64), C.POINTER(C.c_float)], i32),
        "x2_integrate": ([vp, vp, u64, vp, vp], i32), "x2_integrate_device": ([vp, vp, u64, vp, vp], i32),
        "x2_trace_rays": ([vp, vp, u64, vp, vp, vp], i32), "x2_trace_rays_device": ([vp, vp, u64, vp, vp, vp], i32),
        "x2_frame_begin": ([vp, u32], i32), "x2_launch": ([vp, vp, u32], i32), "x2_poll": ([vp, C.POINTER(Completion)], i32),
        "x2_wait": ([vp, i32, C.POINTER(Completion)], i32), "x2_render_frame": ([vp, u32, u32], i32),
        "x2_film_download": ([vp, vp, vp, vp], i32), "x2_film_device": ([vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)], i32),
        "x2_audit": ([vp, vp, C.POINTER(C.c_int64)], i32), "x2_counters_read": ([vp, C.POINTER(Counters)], i32),
        "x2_wavefront_reserve": ([vp, u32], i32), "x2_launch_wavefront": ([vp, vp, u32], i32),
        "x2_render_frame_wavefront": ([vp, u32, u32], i32), "x2_items_download": ([vp, vp, vp, u64], i32),
        "x2_wavefront_info": ([vp, C.POINTER(u32), C.POINTER(u32), C.POINTER(u32)], i32),
        "x2_wavefront_timing": ([vp, i32, vp], i32), "x2_wavefront_queues": ([vp, vp, u32], i32),
        "x2_wavefront_tune": ([vp, C.POINTER(WavefrontShape)], i32), "x2_wavefront_shape_defaults": ([C.POINTER(WavefrontShape)], None),
        "x2_launch_wavefront_static": ([vp, vp, u32, u32, vp, vp, C.POINTER(u64)], i32),
        "x2_render_batch": ([vp, C.POINTER(Request), u32, C.POINTER(Completion)], i32),
        "x2_wavefront_autotune": ([vp, u32, u32, C.POINTER(WavefrontShape), C.POINTER(C.c_float)], i32),
        "x2_scene_set_params": ([vp, vp, vp, vp], i32), "x2_adjoint": ([vp, u32, u32, vp, vp, vp, vp, vp], i32), "x2_adjoint_plain": ([vp, u32, u32, vp, vp, vp, vp, vp], i32),
        "x2_scene_set_texture": ([vp, u32, vp], i32),
        "x2_frame_begin_adaptive": ([vp, u32], i32), "x2_adaptive_step": ([vp, C.c_float, u32, u32, vp, vp, vp], i32),
        "x2_render_adaptive": ([vp, u32, u32, C.c_float, C.POINTER(AdaptiveResult)], i32), "x2_render_adaptive_cellular": ([vp, u32, u32, C.c_float, C.POINTER(AdaptiveResult)], i32),
        "x2_render_adaptive_budget": ([vp, u32, u32, C.c_float, u64, C.POINTER(AdaptiveResult)], i32), "x2_adaptive_planned": ([vp, vp], i32),
        "x2_counters_reset": ([vp], i32), "x2_count_traversal": ([vp, i32], i32),
        "x2_probe_bandwidth": ([vp, u32, u64, u32, C.POINTER(C.c_float)], i32),
        "x2_traversal_counts": ([vp, vp, vp, vp], i32), "x2_traversal_lanes": ([vp, vp], i32), "x2_scene_generate": ([u32, u64, C.POINTER(C.POINTER(SceneDesc)), C.POINTER(Config)], i32),
        "x2_scene_desc_free": ([C.POINTER(SceneDesc)], None),
        "x2_workgrid_options_defaults": ([C.POINTER(WorkGridOptions)], None),
        "x2_workgrid_create": ([u32, u32, u32, C.POINTER(WorkGridOptions), u32, vp, C.POINTER(vp)], i32),
        "x2_workgrid_free": ([vp], None), "x2_workgrid_info": ([vp, vp, vp, vp, C.POINTER(WorkGridOptions)], i32),
        "x2_workgrid_cells": ([vp], u32), "x2_workgrid_total": ([vp], u64), "x2_workgrid_ranges": ([vp, vp, u32], u32),
        "x2_workgrid_cell": ([vp, u32, C.POINTER(u32), C.POINTER(u32), C.POINTER(u32)], i32),
        "x2_workgrid_append": ([vp, u32, vp, u32], i32), "x2_workgrid_claim": ([vp, u32, u32, vp], u32),
        "x2_workgrid_claimable": ([vp, u32], u32), "x2_workgrid_remaining": ([vp, u32], u32), "x2_workgrid_empty": ([vp], u32),
        "x2_workgrid_frontier": ([vp], u32), "x2_workgrid_choose": ([vp, u32, u32], u32),
        "x2_workgrid_seed": ([vp, u32, u32], u32), "x2_workgrid_set_scores": ([vp, vp, u32], i32),
        "x2_workgrid_close": ([vp], None), "x2_workgrid_take": ([vp, u32, vp], u32),
        "x2_render_workgrid": ([vp, vp, u32, C.POINTER(WorkGridResult)], i32), "x2_workgrid_score_film": ([vp, vp, vp], i32),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


def _check(rc):
    if rc != OK:
        raise X2Error(rc, library().x2_last_error().decode())


def _ptr(a):
    return C.c_void_p(a.ctypes.data) if a is not None else C.c_void_p(0)


def config_defaults():
    c = Config()
    library().x2_config_defaults(C.byref(c))
    return c


class Context:
    """One CUDA device and stream (GpuLane's own, async_gpu.h:82)."""

    def __init__(self, device=0):
        self._h = C.c_void_p()
        _check(library().x2_open(device, C.byref(self._h)))
        self.device = device
        self._scenes = weakref.WeakSet()

    @property
    def handle(self):
        return self._h

    def close(self):
        """Frees the context's scenes first: a scene never outlives the context it was loaded on."""
        if self._h:
            for s in list(self._scenes):
                s.free()
            library().x2_close(self._h)
            self._h = C.c_void_p()

    def probe_bandwidth(self, level, nbytes, passes):
        """The device's L2 (level 2) or L1 (level 1) read bandwidth in GB/s (x2_probe_bandwidth)."""
        g = C.c_float()
        _check(library().x2_probe_bandwidth(self._h, level, nbytes, passes, C.byref(g)))
        return g.value

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self, timeout_ms=600000):
        _check(library().x2_synchronize(self._h, timeout_ms))

    def render_batch(self, requests):
        """Many frames in one wavefront launch (x2_render_batch): requests are (Scene, first, count); each scene's
        film then holds its frame. Returns the batch's Completion (samples, errors, device milliseconds)."""
        arr = (Request * len(requests))()
        for i, (scene, first, count) in enumerate(requests):
            arr[i].scene = scene.handle.value
            arr[i].first = first
            arr[i].count = count
        c = Completion()
        _check(library().x2_render_batch(self._h, arr, len(requests), C.byref(c)))
        return c

    def sample_words(self, ids, dims, policy):
        """sample::samplingWord for structured `ids` (IDENTITY_DTYPE) and uint32 `dims` (host arrays)."""
        ids = np.ascontiguousarray(ids, dtype=IDENTITY_DTYPE)
        dims = np.ascontiguousarray(dims, dtype=np.uint32)
        out = np.empty(len(dims), np.uint32)
        _check(library().x2_sample_words(self._h, _ptr(ids), _ptr(dims), len(dims), policy, _ptr(out)))
        return out


IDENTITY_DTYPE = np.dtype([("pixel", "<u4"), ("pad", "<u4"), ("index", "<u8"), ("stream", "<u8"), ("branch", "<u8")])


class SyntheticScene:
    """A seeded synthetic scene made by the library's host generator (x2_scene_generate): its descriptor (owned
    by the library until freed) and the config that goes with it."""

    def __init__(self, config_id, seed=None, generator=None):
        """`generator`: another loaded library exporting x2_scene_generate / x2_scene_desc_free with their
        signatures declared (the oracle's, which compiles the same generator), in place of libx2."""
        self._desc = C.POINTER(SceneDesc)()
        self.config = Config()
        self.config_id = config_id
        self._gen = generator
        if seed is None:  # a config's generator seed is its index + 1; batched requests (200+, 300+) are config 2's
            seed = 3 if 200 <= config_id < 400 else (config_id % 100) + 1
        self.seed = seed
        lib = generator or library()
        rc = lib.x2_scene_generate(config_id, self.seed, C.byref(self._desc), C.byref(self.config))
        if rc != OK:
            raise X2Error(rc, f"x2_scene_generate({config_id}, {self.seed}) failed")

    @property
    def desc(self):
        return self._desc.contents

    @property
    def desc_ptr(self):
        return self._desc

    def arrays(self):
        d = self.desc
        return {
            "vertices": np.ctypeslib.as_array(d.vertices, (d.vertex_count * 3,)).copy(),
            "triangles": np.ctypeslib.as_array(d.triangles, (d.triangle_count * 3,)).copy(),
            "mesh_first": np.ctypeslib.as_array(d.mesh_first, (d.mesh_count + 1,)).copy(),
            "mesh_material": np.ctypeslib.as_array(d.mesh_material, (d.mesh_count,)).copy(),
        }

    def texture(self, k=0):
        """Texture k's texels (height x width x 3, float32), a copy."""
        t = self.desc.textures[k]
        return np.ctypeslib.as_array(t.rgb, (t.height * t.width * 3,)).reshape(t.height, t.width, 3).copy()

    def free(self):
        if self._desc:
            (self._gen or library()).x2_scene_desc_free(self._desc)
            self._desc = C.POINTER(SceneDesc)()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Scene:
    """A scene on the device with its BVH (built on the device at load) and its config."""

    def __init__(self, ctx, desc, config):
        self.ctx = ctx
        self._h = C.c_void_p()
        _check(library().x2_scene_load(ctx.handle, C.byref(desc) if isinstance(desc, SceneDesc) else desc, C.byref(self._h)))
        ctx._scenes.add(self)
        self.set_config(config)

    def set_config(self, config):
        _check(library().x2_config_set(self._h, C.byref(config)))
        self.config = config

    @property
    def handle(self):
        return self._h

    def info(self):
        n, b, t, ms = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_float()
        _check(library().x2_scene_info(self._h, C.byref(n), C.byref(b), C.byref(t), C.byref(ms)))
        return {"bvh_nodes": n.value, "bvh_bytes": b.value, "triangle_bytes": t.value, "build_ms": ms.value}

    def free(self):
        if self._h:
            library().x2_scene_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    # -- per sample: integrate() --
    def integrate(self, pixels, indices):
        """Radiance (rgb + alpha, float64) and SampleStatus of each (pixel, index) sample."""
        pixels = np.asarray(pixels, np.uint32)
        indices = np.asarray(indices, np.uint32)
        pairs = np.ascontiguousarray(np.stack([pixels, indices], axis=1).astype(np.uint32))
        n = len(pixels)
        rgba = np.empty((n, 4), np.float64)
        status = np.empty(n, np.uint32)
        _check(library().x2_integrate(self._h, _ptr(pairs), n, _ptr(rgba), _ptr(status)))
        return rgba, status

    # -- traversal: Backend::trace / visible --
    def trace_rays(self, rays):
        """Closest hit (scene triangle, ~0 for none), its t, and occlusion of [near, far] for (n, 8) float32 rays."""
        rays = np.ascontiguousarray(rays, np.float32)
        n = len(rays)
        tri = np.empty(n, np.uint32)
        t = np.empty(n, np.float32)
        occ = np.empty(n, np.uint32)
        _check(library().x2_trace_rays(self._h, _ptr(rays), n, _ptr(tri), _ptr(t), _ptr(occ)))
        return tri, t, occ

    # -- lane API --
    def frame_begin(self, samples_per_chunk):
        _check(library().x2_frame_begin(self._h, samples_per_chunk))

    def frame_begin_adaptive(self, samples_per_chunk):
        """x2_frame_begin_adaptive: a frame whose film also keeps the odd-index sums."""
        _check(library().x2_frame_begin_adaptive(self._h, samples_per_chunk))

    def adaptive_step(self, target, uniform, size):
        """One adaptive chain step on the current film: (errors [pixels], tile masks [tiles] uint64, stop)."""
        cfg = self.config
        errors = np.empty(cfg.width * cfg.height, np.float32)
        masks = np.empty(((cfg.width + 7) // 8) * ((cfg.height + 7) // 8), np.uint64)
        stop = C.c_uint32()
        _check(library().x2_adaptive_step(self._h, target, uniform, size, _ptr(errors), _ptr(masks), C.byref(stop)))
        return errors, masks, stop.value

    def render_adaptive(self, min_samples, max_samples, target, cellular=False):
        """x2_render_adaptive (cellular: x2_render_adaptive_cellular): an adaptive frame; returns its AdaptiveResult as
        a dict."""
        r = AdaptiveResult()
        f = library().x2_render_adaptive_cellular if cellular else library().x2_render_adaptive
        _check(f(self._h, min_samples, max_samples, target, C.byref(r)))
        return {"passes": r.passes, "converged": bool(r.converged), "samples": r.samples, "milliseconds": r.milliseconds}

    def render_workgrid(self, grid, chunks_per_launch):
        """x2_render_workgrid: a frame fed from a work grid by the GPU broker; returns its WorkGridResult as a dict."""
        r = WorkGridResult()
        _check(library().x2_render_workgrid(self._h, grid._h, chunks_per_launch, C.byref(r)))
        return {k: getattr(r, k) for k, _ in WorkGridResult._fields_}

    def render_adaptive_budget(self, min_samples, max_samples, floor, budget):
        """x2_render_adaptive_budget: a frame by cellular generations under a budget of `budget` samples."""
        r = AdaptiveResult()
        _check(library().x2_render_adaptive_budget(self._h, min_samples, max_samples, floor, budget, C.byref(r)))
        return {"passes": r.passes, "converged": bool(r.converged), "samples": r.samples, "milliseconds": r.milliseconds}

    def score_workgrid(self, grid):
        """x2_workgrid_score_film: the grid's cell scores from this scene's film (set on the grid); returns them."""
        out = np.zeros(grid.cells, np.float32)
        _check(library().x2_workgrid_score_film(self._h, grid._h, _ptr(out)))
        return out

    def adaptive_planned(self):
        cfg = self.config
        planned = np.empty(cfg.width * cfg.height, np.uint32)
        _check(library().x2_adaptive_planned(self._h, _ptr(planned)))
        return planned

    def launch(self, chunks):
        chunks = np.ascontiguousarray(chunks, dtype=CHUNK_DTYPE)
        _check(library().x2_launch(self._h, _ptr(chunks), len(chunks)))

    def render_frame(self, first, count):
        _check(library().x2_render_frame(self._h, first, count))

    # -- wavefront form --
    def wavefront_reserve(self, paths):
        _check(library().x2_wavefront_reserve(self._h, paths))

    def launch_wavefront(self, chunks):
        chunks = np.ascontiguousarray(chunks, dtype=CHUNK_DTYPE)
        _check(library().x2_launch_wavefront(self._h, _ptr(chunks), len(chunks)))

    def render_frame_wavefront(self, first, count):
        _check(library().x2_render_frame_wavefront(self._h, first, count))

    def items(self, n):
        """The last wavefront launch's per-item radiance (n x 4 float32) and SampleStatus."""
        rgba = np.empty((n, 4), np.float32)
        status = np.empty(n, np.uint8)
        _check(library().x2_items_download(self._h, _ptr(rgba), _ptr(status), n))
        return rgba, status

    def launch_wavefront_static(self, d_chunks, count, samples_per_chunk, d_sums, d_counts):
        """The wavefront launch that allocates nothing (x2_launch_wavefront_static): device pointers (ints) to the
        chunks and to the film it adds to; waits; returns the samples rendered."""
        done = C.c_uint64()
        _check(library().x2_launch_wavefront_static(self._h, C.c_void_p(d_chunks), count, samples_per_chunk, C.c_void_p(d_sums),
                                                    C.c_void_p(d_counts), C.byref(done)))
        return done.value

    def wavefront_timing(self, on=None):
        """Switch per-kernel timing (diagnostic) and return the last timed launch's milliseconds by kernel."""
        ms = np.zeros(5, np.float32)
        _check(library().x2_wavefront_timing(self._h, -1 if on is None else int(bool(on)), _ptr(ms)))
        return dict(zip(("logic", "extend", "shade", "shadow", "film"), ms.tolist()))

    def wavefront_tune(self, **shape):
        """Launch shape of the wavefront kernels (x2_wavefront_shape fields by name; the others keep their defaults).
        Returns the shape set, as a dict."""
        s = wavefront_shape_defaults()
        for k, v in shape.items():
            if k not in WavefrontShape.FIELDS:
                raise ValueError("no wavefront shape field %r" % k)
            setattr(s, k, int(v))
        _check(library().x2_wavefront_tune(self._h, C.byref(s)))
        return s.as_dict()

    def set_params(self, albedo=None, radiance=None, roughness=None):
        """The differentiable parameters (x2_scene_set_params): each material's diffuse colour (n x 3), each light's
        radiance (n x 3) and each material's roughness (n), or None to leave a set."""
        a = None if albedo is None else np.ascontiguousarray(albedo, np.float32)
        r = None if radiance is None else np.ascontiguousarray(radiance, np.float32)
        g = None if roughness is None else np.ascontiguousarray(roughness, np.float32)
        _check(library().x2_scene_set_params(self._h, _ptr(a), _ptr(g), _ptr(r)))

    def set_texture(self, texture, rgb):
        """x2_scene_set_texture: texture `texture`'s texels (height x width x 3 floats) set in place."""
        a = np.ascontiguousarray(rgb, np.float32)
        _check(library().x2_scene_set_texture(self._h, texture, _ptr(a)))

    def adjoint(self, first, count, d_dloss_dimage, d_albedo_grad, d_radiance_grad, d_roughness_grad=None, plain=False,
                d_texture_grad=None):
        """x2_adjoint on device pointers (ints): adds dL/dalbedo, dL/dradiance and (when given) dL/droughness and
        dL/dtexel for samples [first, first + count) of every pixel, given dL/dimage (3 floats a pixel). plain: the
        replay in the plain megakernel's form (x2_adjoint_plain)."""
        f = library().x2_adjoint_plain if plain else library().x2_adjoint
        _check(f(self._h, first, count, C.c_void_p(d_dloss_dimage), C.c_void_p(d_albedo_grad), C.c_void_p(d_roughness_grad),
                 C.c_void_p(d_radiance_grad), C.c_void_p(d_texture_grad)))

    def wavefront_autotune(self, tiles=0, spp=None):
        """Time the wavefront launch shapes on `tiles` evenly spaced tiles (0: all) at `spp` samples (default: the
        config's), set the fastest and return (shape dict, its milliseconds). Leaves the film reset."""
        best = WavefrontShape()
        ms = C.c_float()
        _check(library().x2_wavefront_autotune(self._h, tiles, spp or self.config.spp, C.byref(best), C.byref(ms)))
        return best.as_dict(), ms.value

    def wavefront_queues(self):
        """The last timed launch's per-iteration queue sizes as an (iterations, 2) array: rays extended, shadow rays."""
        n = self.wavefront_info()["iterations"]
        sizes = np.zeros(2 * min(n, 4096), np.uint32)
        _check(library().x2_wavefront_queues(self._h, _ptr(sizes), sizes.size))
        return sizes.reshape(-1, 2)

    def wavefront_info(self):
        p, r, i = C.c_uint32(), C.c_uint32(), C.c_uint32()
        _check(library().x2_wavefront_info(self._h, C.byref(p), C.byref(r), C.byref(i)))
        return {"paths": p.value, "records_per_path": r.value, "iterations": i.value}

    def poll(self):
        c = Completion()
        r = library().x2_poll(self._h, C.byref(c))
        if r < 0:
            _check(-r)
        return c if r == 1 else None

    def wait(self, timeout_ms=600000):
        c = Completion()
        _check(library().x2_wait(self._h, timeout_ms, C.byref(c)))
        return c

    def film_tensors(self, odd=False):
        """The film in place on the device as torch tensors (no copy; x2_film_device): FP64 sums (pixels x 4), the odd
        sums (or None) and the counts as int32 (the library's uint32 counts, equal while below 2^31). The library writes
        them on its own stream: call wait() before reading them and synchronise torch's work before the next launch."""
        import torch

        sums, odd_p, counts = C.c_void_p(), C.c_void_p(), C.c_void_p()
        _check(library().x2_film_device(self._h, C.byref(sums), C.byref(odd_p), C.byref(counts)))
        p = self.config.width * self.config.height
        dev = "cuda:%d" % self.ctx.device

        def view(ptr, shape, typestr):
            arr = type("DeviceArray", (), {})()
            arr.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (ptr.value, False), "version": 3,
                                            "strides": None}
            return torch.as_tensor(arr, device=dev)

        out_odd = view(odd_p, (p, 4), "<f8") if odd and odd_p.value else None
        return view(sums, (p, 4), "<f8"), out_odd, view(counts, (p,), "<i4")

    def film(self, odd=False, out=None):
        """The film on the host (x2_film_download; waits): FP64 sums (pixels x 4), with `odd` the odd-index sums, and
        the uint32 counts. `out`, a (sums, counts) or (sums, odd, counts) tuple of C-contiguous arrays of those shapes
        and types, receives them instead of new arrays: arrays kept across frames (pinned ones copy fastest) spare each
        frame the allocation and first touch of the film's pages."""
        p = self.config.width * self.config.height
        if out is not None:
            sums, counts = out[0], out[-1]
            o = out[1] if odd else None
            for arr, shape, dt in ((sums, (p, 4), np.float64), (counts, (p,), np.uint32), (o, (p, 4), np.float64)):
                if arr is not None and (arr.shape != shape or arr.dtype != dt or not arr.flags["C_CONTIGUOUS"]):
                    raise ValueError("film out arrays must be C-contiguous %s of %s" % (shape, np.dtype(dt).name))
        else:
            sums = np.empty((p, 4), np.float64)
            counts = np.empty(p, np.uint32)
            o = np.empty((p, 4), np.float64) if odd else None
        _check(library().x2_film_download(self._h, _ptr(sums), _ptr(o), _ptr(counts)))
        return (sums, o, counts) if odd else (sums, counts)

    def audit(self, expected=None):
        """The per-pixel sample-count audit (async_render.h:1010-1040); raises X2Error(EAUDIT) on a mismatch."""
        bad = C.c_int64()
        e = None if expected is None else np.ascontiguousarray(expected, np.uint32)
        _check(library().x2_audit(self._h, _ptr(e), C.byref(bad)))

    def counters(self):
        c = Counters()
        _check(library().x2_counters_read(self._h, C.byref(c)))
        return c.as_dict()

    def reset_counters(self):
        _check(library().x2_counters_reset(self._h))

    def count_traversal(self, on):
        """Counting mode: following launches count node visits and triangle tests (never time them)."""
        _check(library().x2_count_traversal(self._h, 1 if on else 0))

    def traversal_counts(self):
        """Node visits and triangle tests of the launches made in counting mode, by ray kind."""
        r, n, t = (C.c_uint64 * 2)(), (C.c_uint64 * 2)(), (C.c_uint64 * 2)()
        lanes = (C.c_uint64 * 12)()
        _check(library().x2_traversal_lanes(self._h, lanes))
        _check(library().x2_traversal_counts(self._h, r, n, t))
        names = ("steps", "live_lanes", "node_steps", "node_lanes", "tri_steps", "tri_lanes")
        return {kind: {"rays": r[k], "nodes": n[k], "triangles": t[k], "lanes": {nm: lanes[6 * k + j] for j, nm in enumerate(names)}}
                for k, kind in enumerate(("closest", "any"))}


CHUNK_DTYPE = np.dtype([("tile", "<u4"), ("first", "<u4"), ("count", "<u4"), ("cell", "<u4")])


def image(sums, counts, width, height):
    """The film's pixel values: (sum over samples) / count, rgba, as the reference's merge does."""
    c = np.maximum(counts, 1).astype(np.float64)[:, None]
    return (sums / c).reshape(height, width, 4)


def workgrid_options(**kw):
    """The work grid's options (x2_workgrid_options_defaults), with the given fields changed."""
    o = WorkGridOptions()
    library().x2_workgrid_options_defaults(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class WorkGrid:
    """The work grid (x2_workgrid_*): cells handing out their chunks through one cursor each, the frontier, the
    cellular choice and the broker; host-side."""

    def __init__(self, width, height, spp, options=None, empty=False, viewport=None):
        self.options = options if options is not None else workgrid_options()
        view = None if viewport is None else np.ascontiguousarray(viewport, np.int32)
        h = C.c_void_p()
        _check(library().x2_workgrid_create(width, height, spp, C.byref(self.options), int(bool(empty)),
                                            _ptr(view) if view is not None else None, C.byref(h)))
        self._h = h

    def free(self):
        if self._h:
            library().x2_workgrid_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    @property
    def cells(self):
        return library().x2_workgrid_cells(self._h)

    @property
    def total(self):
        return library().x2_workgrid_total(self._h)

    def ranges(self):
        n = library().x2_workgrid_ranges(self._h, None, 0)
        out = np.zeros(2 * max(n, 1), np.uint32)
        library().x2_workgrid_ranges(self._h, _ptr(out), n)
        return [(int(out[2 * k]), int(out[2 * k + 1])) for k in range(n)]

    def cell(self, i):
        v = [C.c_uint32() for _ in range(3)]
        _check(library().x2_workgrid_cell(self._h, i, *[C.byref(x) for x in v]))
        return dict(zip(("tiles", "published", "taken"), (x.value for x in v)))

    def append(self, cell, chunks):
        chunks = np.ascontiguousarray(chunks, dtype=CHUNK_DTYPE)
        _check(library().x2_workgrid_append(self._h, cell, _ptr(chunks), len(chunks)))

    def claim(self, cell, n):
        out = np.zeros(max(n, 1), CHUNK_DTYPE)
        got = library().x2_workgrid_claim(self._h, cell, n, _ptr(out))
        return out[:got]

    def claimable(self, cell):
        return library().x2_workgrid_claimable(self._h, cell)

    def remaining(self, cell):
        return library().x2_workgrid_remaining(self._h, cell)

    def empty(self):
        return bool(library().x2_workgrid_empty(self._h))

    def frontier(self):
        return library().x2_workgrid_frontier(self._h)

    def choose(self, current, salt):
        return library().x2_workgrid_choose(self._h, current, salt)

    def seed(self, worker, workers):
        return library().x2_workgrid_seed(self._h, worker, workers)

    def set_scores(self, scores):
        scores = np.ascontiguousarray(scores, np.float32)
        _check(library().x2_workgrid_set_scores(self._h, _ptr(scores), len(scores)))

    def close(self):
        library().x2_workgrid_close(self._h)

    def take(self, want):
        """The broker's next launch: up to `want` chunks (x2_workgrid_take)."""
        out = np.zeros(max(want, 1), CHUNK_DTYPE)
        got = library().x2_workgrid_take(self._h, want, _ptr(out))
        return out[:got]
