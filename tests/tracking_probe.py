"""Image means of the participating medium (config 3) by tracking and by the march, in the diagnostic build of
libx2 (libx2diag.so), run as its own process because the x2 module loads one library a process. Test infrastructure
for tests/test_gpu_tracking.py.

    python tests/tracking_probe.py <out.json>

Over the pixels of the fixture tiles (tests/golden/rmse_c3.npz): the tracked image's mean at the configured steps over
16,384 samples a pixel, and the march's at steps 16 times finer over 4,096: as the reference computes it (diagnostic
mode 0) and with the single scattering's distance samples taking their pair's equi-angular light point (mode 4,
x2_diag.h).
"""
import ctypes as C
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "xpu2-foundation_b200"))
sys.path.insert(0, HERE)
os.environ["X2_LIBRARY"] = os.path.join(ROOT, "xpu2-foundation_b200", "x2", "libx2diag.so")

import rmse_lib  # noqa: E402
import x2  # noqa: E402


def image_mean(ctx, pixels, estimator, finer, n):
    s = x2.SyntheticScene(3)
    cfg = s.config
    cfg.volume_estimator = estimator
    cfg.inv_volume_quality /= finer
    cfg.inv_volume_shadow_quality /= finer
    scene = x2.Scene(ctx, s.desc, cfg)
    sums = np.zeros((len(pixels), 3))
    for first in range(0, n, 1024):
        p = np.repeat(pixels, 1024)
        idx = np.tile(np.arange(first, first + 1024, dtype=np.uint32), len(pixels))
        rgba, status = scene.integrate(p, idx)
        assert (status == x2.DONE).all()
        sums += rgba[:, :3].reshape(len(pixels), 1024, 3).sum(1)
    scene.free()
    s.free()
    return float((sums / n).mean())


def main(dst):
    lib = x2.library()
    lib.x2_diag_set.argtypes = [C.c_int, C.c_void_p, C.c_uint32]
    lib.x2_diag_set.restype = C.c_int
    ctx = x2.Context(0)
    f = np.load(os.path.join(HERE, "golden", "rmse_c3.npz"))
    base = x2.SyntheticScene(3)
    pixels = rmse_lib.tile_pixels(f["tiles"], base.config.width, base.config.height)[f["live"]].astype(np.uint32)
    out = {}
    assert lib.x2_diag_set(0, None, 0) == 0
    out["tracked"] = image_mean(ctx, pixels, 1, 1, 16384)
    out["march_16"] = image_mean(ctx, pixels, 0, 16, 4096)
    assert lib.x2_diag_set(4, None, 0) == 0
    out["march_16_shared_pivot"] = image_mean(ctx, pixels, 0, 16, 4096)
    assert lib.x2_diag_set(0, None, 0) == 0
    with open(dst, "w") as fh:
        json.dump(out, fh)


if __name__ == "__main__":
    main(sys.argv[1])
