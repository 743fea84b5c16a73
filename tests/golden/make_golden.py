"""Generates the golden fixtures under tests/golden/ from the reference itself.

Run here (where the reference's sources exist and oracle/_ref/libx2ref.so was compiled from them):
    python tests/golden/make_golden.py
Outputs (small, committed):
  sampler_words.npz   samplingWord of seeded identities x dimensions 0..40 (and 16+bounce*256+k stream draws)
                      under policies 0, 3 and 15, from the reference's sample_stream.h compiled from source.
  philox_kat.json     the three Philox4x32-10 known-answer vectors of the reference's sample_fixture.h:17-20 and
                      its Sobol first-eight-points table, qmc_fixture.h:14-15 (copied as data, by hand, from those
                      test files).
  radiance_c0.npz     per-sample Radiance (rgb, alpha) and SampleStatus of seeded (pixel, index) samples of the
  radiance_c108.npz   closed box and of the config-1 scene scaled down by 8, from the reference's integratePaths.
  radiance_c33.npz    the same for the participating medium of config 3, shrunk (a 32^3 grid in the closed box).
  radiance_c44.npz    the same for the differentiable scene shrunk (config 44: a textured heightfield, UsdUVTexture).
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import oracle_lib  # noqa: E402
from oracle_lib import x2  # noqa: E402


def sampler_words():
    ids = oracle_lib.random_identities(512, seed=7)
    dims = np.concatenate([np.arange(41), 16 + 256 * np.arange(1, 4)[:, None].repeat(4, 1).ravel() + np.tile(np.arange(4), 3)])
    rows_ids = np.repeat(ids, len(dims))
    rows_dims = np.tile(dims, len(ids)).astype(np.uint32)
    out = {}
    for policy in (0, 3, 15):
        out[f"p{policy}"] = oracle_lib.reference_sampling_words(rows_ids, rows_dims, policy)
    np.savez_compressed(os.path.join(HERE, "sampler_words.npz"), ids=rows_ids, dims=rows_dims, **out)


def philox_kat():
    kat = {
        "philox": [
            {"counter": [0, 0, 0, 0], "key": [0, 0], "out": [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]},
            {"counter": [0xFFFFFFFF] * 4, "key": [0xFFFFFFFF] * 2, "out": [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]},
            {"counter": [0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], "key": [0xA4093822, 0x299F31D0],
             "out": [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]},
        ],
        "sobol_first8": [[0, 4, 6, 2, 3, 7, 5, 1], [0, 4, 2, 6, 3, 7, 1, 5], [0, 4, 2, 6, 5, 1, 7, 3], [0, 4, 2, 6, 7, 3, 5, 1]],
        "word_5_3_1_0_dim0": 0xF05DB22F,
    }
    with open(os.path.join(HERE, "philox_kat.json"), "w") as f:
        json.dump(kat, f, indent=1)


def radiance(config_id, n, seed):
    s = x2.SyntheticScene(config_id)
    ref = oracle_lib.Reference(s)
    pixels, indices = oracle_lib.sample_pairs(s.config, n, seed)
    rgba, status = ref.integrate(pixels, indices)
    np.savez_compressed(os.path.join(HERE, f"radiance_c{config_id}.npz"), pixels=pixels, indices=indices, rgba=rgba, status=status)
    return rgba, status


if __name__ == "__main__":
    if not oracle_lib.have_reference():
        sys.exit("oracle/_ref/libx2ref.so is missing: build it with `make -f oracle/Makefile`")
    sampler_words()
    philox_kat()
    print("c0", radiance(0, 4096, 11)[1].tolist().count(0), "done of 4096")
    print("c108", radiance(108, 2048, 12)[1].tolist().count(0), "done of 2048")
    print("c33", radiance(33, 2048, 13)[1].tolist().count(0), "done of 2048")
    print("c44", radiance(44, 4096, 14)[1].tolist().count(0), "done of 4096")
    print("ok")
