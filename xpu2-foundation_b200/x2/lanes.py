"""Frames split across GPUs: one process a GPU, each rendering a share of the frame's samples, the films summed at
frame end and audited once.

The reference splits a frame the same two ways. A share of a frame is a contiguous range of its sample indices
(`sampleFirst`, `sampleCount`; a pixel's expected count in a share is `min(sampleCount, spp - sampleFirst)`,
xi/async_render.h:1019-1021), so the shares' films add up to the whole frame's, sample for sample. Lanes' films are
summed element by element (sums, odd sums, counts; GpuLane::addFollowers, xi/async_gpu.h:1641-1660) and the merged
counts are audited against the samples planned for each pixel (xi/async_render.h:1022-1031).

Here the sum runs as one reduce a buffer over torch.distributed: NCCL between GPUs, gloo for the CPU tests. Every
rank makes the same collective calls in the same order.
"""
import numpy as np

from . import X2Error, EAUDIT


def share(rank, world, spp):
    """Rank `rank`'s share of a frame of `spp` samples a pixel: (first sample index, sample count), contiguous ranges
    covering [0, spp) once, the first `spp % world` ranks taking one sample more."""
    if not 0 <= rank < world:
        raise ValueError("rank %d outside a world of %d" % (rank, world))
    base, extra = divmod(spp, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def expected_counts(pixels, spp, first, count):
    """The per-pixel sample count a share [first, first+count) of a uniform frame of `spp` samples must leave."""
    n = 0 if spp <= first else min(count, spp - first)
    return np.full(pixels, n, np.uint32)


def audit(counts, expected):
    """Index of the first pixel whose count differs from the plan, or -1; a pixel with no samples planned may hold
    none."""
    counts = np.asarray(counts)
    bad = np.flatnonzero(counts.astype(np.int64) != np.asarray(expected, np.int64))
    return int(bad[0]) if bad.size else -1


def merge(sums, counts, odd=None, dst=0, group=None, device=None):
    """Sum the ranks' films into rank `dst` (float64 sums and odd sums, uint32 counts as int64); returns the merged
    numpy arrays on `dst` and None elsewhere. `device` is where the reduce runs: a CUDA device for NCCL, None (CPU)
    for gloo."""
    import torch
    import torch.distributed as dist

    bufs = [torch.from_numpy(np.ascontiguousarray(sums, np.float64)), torch.from_numpy(np.asarray(counts).astype(np.int64))]
    if odd is not None:
        bufs.append(torch.from_numpy(np.ascontiguousarray(odd, np.float64)))
    if device is not None:
        bufs = [b.to(device) for b in bufs]
    for b in bufs:
        dist.reduce(b, dst, op=dist.ReduceOp.SUM, group=group)
    if dist.get_rank(group) != dst:
        return None
    out = [b.cpu().numpy() for b in bufs]
    out[1] = out[1].astype(np.uint32)
    return tuple(out) if odd is not None else (out[0], out[1])


def merge_and_audit(sums, counts, spp, odd=None, dst=0, group=None, device=None):
    """`merge`, then the whole frame's audit on `dst`: every pixel holds exactly `spp` samples. Raises X2Error(EAUDIT)
    on the first pixel that does not."""
    merged = merge(sums, counts, odd, dst, group, device)
    if merged is None:
        return None
    bad = audit(merged[1], expected_counts(len(merged[1]), spp, 0, spp))
    if bad >= 0:
        raise X2Error(EAUDIT, "Sample audit failure at pixel %d: %d" % (bad, int(merged[1][bad])))
    return merged


def merge_device(scene, odd=False, group=None):
    """Sum the ranks' films in place on their devices: every rank's scene film (sums, counts and, with `odd`, the odd
    sums) becomes the sum over the group, with no copy through the host. An all-reduce a buffer, NCCL between GPUs (gloo
    stages through the host in the single-GPU tests). Waits for the scene's launches first and for the reduces after."""
    import torch
    import torch.distributed as dist

    scene.wait()
    sums, odd_t, counts = scene.film_tensors(odd)
    for b in (sums, counts) + ((odd_t,) if odd_t is not None else ()):
        dist.all_reduce(b, op=dist.ReduceOp.SUM, group=group)
    torch.cuda.synchronize(sums.device)


def merge_and_audit_device(scene, spp, odd=False, group=None):
    """`merge_device`, then the merged film's audit on the device (x2_audit): every pixel holds exactly `spp` samples.
    Raises X2Error(EAUDIT) on the first pixel that does not, on every rank (each holds the merged film)."""
    merge_device(scene, odd, group)
    pixels = scene.config.width * scene.config.height
    scene.audit(np.full(pixels, spp, np.uint32))


def resolve(sums, counts):
    """Pixel values: sum / count per channel as float32, black where a pixel holds no samples."""
    c = np.asarray(counts, np.float64)[:, None]
    return np.where(c > 0, np.asarray(sums) / np.maximum(c, 1), 0.0).astype(np.float32)
