"""The wavefront launch that allocates nothing (x2_launch_wavefront_static), against the allocating one.

It is for callers that cannot call cudaMalloc (device memory held by another allocator, or no implicit device
synchronisation allowed): its scratch is a static device array, and the caller brings the chunks and the film in its
own device memory. Two calls in a row must each give the film the allocating entry point gives for the same chunks,
within the parity tolerance — the second call reuses the array the first left behind. This file is collected last so
that a failure here comes after every other test has run; it also passes alone in a fresh process.
"""
import numpy as np
import pytest

from oracle_lib import x2

pytestmark = pytest.mark.gpu
RTOL, ATOL = 1e-4, 1e-6


def test_static_scratch_entry_matches_allocating_entry(ctx):
    import torch

    s = x2.SyntheticScene(108)
    cfg = s.config
    scene = x2.Scene(ctx, s.desc, cfg)
    tiles = ((cfg.width + 7) // 8) * ((cfg.height + 7) // 8)
    spc = 3
    chunks = np.zeros(tiles, x2.CHUNK_DTYPE)
    chunks["tile"], chunks["first"], chunks["count"] = np.arange(tiles), 7, spc
    assert tiles * 64 * spc <= 1 << 20

    scene.frame_begin(spc)
    scene.launch_wavefront(chunks)
    scene.wait()
    want_sums, want_counts = scene.film()

    pixels = cfg.width * cfg.height
    dev = torch.device("cuda", 0)
    d_chunks = torch.from_numpy(chunks.view(np.uint32).copy()).to(dev)
    d_sums = torch.zeros(pixels * 4, dtype=torch.float64, device=dev)
    d_counts = torch.zeros(pixels, dtype=torch.int32, device=dev)
    for call in range(2):
        d_sums.zero_()
        d_counts.zero_()
        torch.cuda.synchronize()
        done = scene.launch_wavefront_static(d_chunks.data_ptr(), tiles, spc, d_sums.data_ptr(), d_counts.data_ptr())
        assert done == pixels * spc, call
        got_counts = d_counts.cpu().numpy().astype(np.uint32)
        got_sums = d_sums.cpu().numpy().reshape(pixels, 4)
        assert np.array_equal(got_counts, want_counts), call
        assert np.allclose(got_sums, want_sums, rtol=RTOL, atol=ATOL), call


def _static_film(scene, chunks, spc, pixels):
    import torch

    dev = torch.device("cuda", 0)
    d_chunks = torch.from_numpy(chunks.view(np.uint32).copy()).to(dev)
    d_sums = torch.zeros(pixels * 4, dtype=torch.float64, device=dev)
    d_counts = torch.zeros(pixels, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    done = scene.launch_wavefront_static(d_chunks.data_ptr(), len(chunks), spc, d_sums.data_ptr(), d_counts.data_ptr())
    return done, d_sums.cpu().numpy().reshape(pixels, 4), d_counts.cpu().numpy().astype(np.uint32)


def test_static_scratch_entry_short_chunks_ragged_image(ctx):
    """Chunks of 1..samples_per_chunk samples over an image whose edge tiles are partial, and one chunk whose count is
    above samples_per_chunk (clamped on the device to samples_per_chunk), against the allocating entry given the
    clamped chunks."""
    s = x2.SyntheticScene(108)
    cfg = s.config
    cfg.width, cfg.height = 250, 130
    scene = x2.Scene(ctx, s.desc, cfg)
    tiles = ((cfg.width + 7) // 8) * ((cfg.height + 7) // 8)
    spc = 4
    chunks = np.zeros(tiles, x2.CHUNK_DTYPE)
    chunks["tile"] = np.arange(tiles)
    chunks["first"] = np.arange(tiles) % 5
    chunks["count"] = 1 + np.arange(tiles) % spc
    over = chunks.copy()
    over["count"][17] = spc + 9
    want_chunks = over.copy()
    want_chunks["count"][17] = spc
    scene.frame_begin(spc)
    scene.launch_wavefront(want_chunks)
    scene.wait()
    want_sums, want_counts = scene.film()
    pixels = cfg.width * cfg.height
    for call in range(2):
        done, sums, counts = _static_film(scene, over, spc, pixels)
        assert done == int(want_counts.sum()), call
        assert np.array_equal(counts, want_counts), call
        assert np.allclose(sums, want_sums, rtol=RTOL, atol=ATOL), call


def test_static_scratch_entry_rejects_unadmitted_configs(ctx):
    """More light records a vertex than the static scratch holds, or more than one BSDF sample: X2_EINVAL."""
    import torch

    s = x2.SyntheticScene(0)
    dev = torch.device("cuda", 0)
    d = torch.zeros(16, dtype=torch.float64, device=dev)
    for field, value in (("light_samples", 33), ("bsdf_samples", 2)):
        cfg = x2.SyntheticScene(0).config
        setattr(cfg, field, value)
        scene = x2.Scene(ctx, s.desc, cfg)
        with pytest.raises(x2.X2Error) as e:
            scene.launch_wavefront_static(d.data_ptr(), 1, 1, d.data_ptr(), d.data_ptr())
        assert e.value.code == x2.EINVAL, field


def test_static_scratch_entry_rejects_oversized_calls(ctx):
    import torch

    s = x2.SyntheticScene(0)
    scene = x2.Scene(ctx, s.desc, s.config)
    dev = torch.device("cuda", 0)
    d = torch.zeros(16, dtype=torch.float64, device=dev)
    with pytest.raises(x2.X2Error) as e:
        scene.launch_wavefront_static(d.data_ptr(), 20000, 1, d.data_ptr(), d.data_ptr())  # 20000 x 64 > 2^20 items
    assert e.value.code == x2.EINVAL
