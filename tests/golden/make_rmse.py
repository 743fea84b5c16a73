"""Generates the image-error fixtures under tests/golden/ (rmse_c*.npz) from the reference itself.

For each benchmark configuration a seeded set of 8x8 tiles is rendered twice by the reference's integratePaths
compiled from source (oracle/_ref/libx2ref.so), on host threads, with FP64 film sums:
  ref   the converged image: 16,384 samples a pixel, sample indices [2^20, 2^20 + 16384) so that they share no
        sample with the configuration's own render;
  cpu   the configuration's own render of those tiles: samples [0, spp) of its frame.
The GPU test (tests/test_gpu_rmse.py) renders the same tiles at the configuration's spp and states the image RMSE of
both forms against `ref`; `cpu` is the reference's own image of those samples (its RMSE is the one to equal).

Configurations and tile counts (the reference CPU integrator's cost decides them; a few minutes each on 8 cores):
  0   the closed box (256x256, 16 spp)                         64 tiles
  1   the 12.3M-triangle field (1920x1080, 64 spp)              24 tiles
  3   the participating medium (512x512, 256 spp)               6 tiles
  4   the differentiable scene, primal (512x512, 32 spp)       24 tiles
  2   requests 200, 203, 207, 211 of the batch (own sizes)      6 tiles each

Run here (the reference's sources exist and the oracle was compiled from them):
    python tests/golden/make_rmse.py [config ...]
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import oracle_lib  # noqa: E402
from oracle_lib import x2  # noqa: E402

REF_SPP = 16384
REF_FIRST = 1 << 20
PLAN = {0: [(0, 64)], 1: [(1, 24)], 3: [(3, 6)], 4: [(4, 24)], 2: [(200, 6), (203, 6), (207, 6), (211, 6)]}


def tiles_of(cfg, n, seed):
    tiles = ((cfg.width + 7) // 8) * ((cfg.height + 7) // 8)
    return np.sort(np.random.default_rng(seed).permutation(tiles)[:n]).astype(np.uint32)


def make(scene_id, n_tiles, threads):
    s = x2.SyntheticScene(scene_id)
    cfg = s.config
    ref = oracle_lib.Reference(s)
    tiles = tiles_of(cfg, n_tiles, 1000 + scene_id)
    t0 = time.time()
    rc, sums, counts = ref.render_tiles_film(tiles, REF_FIRST, REF_SPP, threads)
    ref_s = time.time() - t0
    assert rc == 0, rc
    rc2, csums, ccounts = ref.render_tiles_film(tiles, 0, cfg.spp, threads)
    assert rc2 == 0, rc2
    ref.close()
    live = counts > 0
    assert np.array_equal(live, ccounts > 0)
    image = np.where(live[..., None], sums[..., :3] / np.maximum(counts, 1)[..., None], 0.0)
    cpu = np.where(live[..., None], csums[..., :3] / np.maximum(ccounts, 1)[..., None], 0.0)
    path = os.path.join(HERE, f"rmse_c{scene_id}.npz")
    np.savez_compressed(path, scene=scene_id, tiles=tiles, ref=image.astype(np.float32), cpu=cpu, live=live, ref_spp=REF_SPP,
                        ref_first=REF_FIRST, spp=cfg.spp, ref_seconds=ref_s, threads=threads)
    rmse = float(np.sqrt(np.mean((cpu[live] - image[live]) ** 2)))
    print(f"scene {scene_id}: {len(tiles)} tiles, reference {REF_SPP} spp in {ref_s:.0f} s; CPU {cfg.spp}-spp RMSE {rmse:.5g}", flush=True)


def main():
    which = [int(a) for a in sys.argv[1:]] or list(PLAN)
    threads = os.cpu_count() or 1
    for c in which:
        for scene_id, n in PLAN[c]:
            make(scene_id, n, threads)


if __name__ == "__main__":
    main()
