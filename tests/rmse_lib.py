"""Image error against the reference's converged renders (tests/golden/rmse_c*.npz, made by
tests/golden/make_rmse.py from the reference integrator at 16,384 samples a pixel, FP64 film sums).

`measure(ctx, path)` renders the fixture's tiles at its configuration's spp through the lane API, in the wavefront form
and with the plain megakernel, and returns the RMSE of each against the converged image, beside the RMSE of the
reference's own render of the same samples (`cpu`). All three images are of the same sample identities, so the three
RMSEs agree up to the 1e-4 per-sample tolerance; the wavefront and plain images are equal.
"""
import glob
import os

import numpy as np

import x2

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def fixtures():
    return sorted(glob.glob(os.path.join(GOLDEN, "rmse_c*.npz")), key=lambda p: int(os.path.basename(p)[6:-4]))


def tile_pixels(tiles, width, height):
    """Pixel of each (tile, position) of 8x8 tiles, row-major within a tile; -1 past the frame's edge."""
    tiles = np.asarray(tiles, np.int64)[:, None]
    pos = np.arange(64)[None, :]
    tx = (width + 7) // 8
    x = (tiles % tx) * 8 + pos % 8
    y = (tiles // tx) * 8 + pos // 8
    return np.where((x < width) & (y < height), y * width + x, -1)


def render_tiles(scene, tiles, spp, wavefront):
    cfg = scene.config
    chunks = np.zeros(len(tiles), x2.CHUNK_DTYPE)
    chunks["tile"], chunks["first"], chunks["count"] = tiles, 0, spp
    scene.frame_begin(spp)
    (scene.launch_wavefront if wavefront else scene.launch)(chunks)
    done = scene.wait()
    sums, counts = scene.film()
    px = tile_pixels(tiles, cfg.width, cfg.height)
    live = px >= 0
    img = np.zeros(px.shape + (3,))
    c = counts[px[live]]
    if not (c == spp).all():
        raise AssertionError("sample counts of the rendered tiles differ from their spp")
    img[live] = sums[px[live], :3] / c[:, None]
    return img, done.milliseconds


def rmse(a, b, live):
    return float(np.sqrt(np.mean((a[live] - b[live]) ** 2)))


def measure(ctx, path):
    f = np.load(path)
    scene_id = int(f["scene"])
    s = x2.SyntheticScene(scene_id)
    scene = x2.Scene(ctx, s.desc, s.config)
    spp = int(f["spp"])
    tiles = f["tiles"]
    live = f["live"]
    ref = f["ref"].astype(np.float64)
    out = {"scene": scene_id, "tiles": int(len(tiles)), "pixels": int(live.sum()), "spp": spp, "ref_spp": int(f["ref_spp"]),
           "triangles": int(s.desc.triangle_count)}
    images = {}
    for form in ("wavefront", "plain"):
        images[form], ms = render_tiles(scene, tiles, spp, form == "wavefront")
        out[form] = {"rmse": rmse(images[form], ref, live), "ms": ms}
    out["cpu_rmse"] = rmse(f["cpu"], ref, live)
    out["forms_equal"] = bool(np.array_equal(images["wavefront"], images["plain"]))
    d = np.abs(images["wavefront"] - f["cpu"])[live]
    out["max_abs_diff_vs_cpu"] = float(d.max())
    inside = d <= 1e-4 * np.abs(f["cpu"][live]) + 1e-6
    out["frac_within_1e-4_vs_cpu"] = float(np.mean(inside))
    # The pixels (frame indices) with a channel outside 1e-4 of the reference's render of the same samples.
    frame_pixels = tile_pixels(tiles, s.config.width, s.config.height)[live]
    out["pixels_outside_1e-4"] = [int(v) for v in frame_pixels[~inside.all(axis=1)]]
    # The converged image's own error (its samples' variance over 16,384): the floor under every RMSE stated here.
    out["ref_mean"] = float(ref[live].mean())
    scene.free()
    s.free()
    return out
