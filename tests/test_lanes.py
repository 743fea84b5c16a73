"""Frames split across ranks (x2.lanes): shares of the sample range, the films' sum-reduce and the merged audit.

Two gloo ranks on the CPU each render their share of a frame with the oracle, the films are merged on rank 0 and
must equal the oracle's film of the whole frame rendered in one piece, and the audit must pass; a planted missing
sample on rank 1 must make the merged audit fail. This is the host logic the multi-GPU bench runs over NCCL.
"""
import json
import os
import socket

import numpy as np
import pytest

from oracle_lib import Reference, have_reference, x2
from x2 import lanes

CONFIG, SPP = 108, 3


def test_shares_cover_the_frame_once():
    for spp in (1, 3, 16, 64, 257):
        for world in (1, 2, 3, 4, 8):
            got = [lanes.share(r, world, spp) for r in range(world)]
            assert got[0][0] == 0
            for (f0, c0), (f1, _) in zip(got, got[1:]):
                assert f0 + c0 == f1
            assert sum(c for _, c in got) == spp
            assert max(c for _, c in got) - min(c for _, c in got) <= 1
    with pytest.raises(ValueError):
        lanes.share(2, 2, 8)


def test_expected_counts_and_audit():
    e = lanes.expected_counts(10, 16, 12, 8)
    assert (e == 4).all()
    assert (lanes.expected_counts(10, 16, 16, 8) == 0).all()
    c = e.copy()
    assert lanes.audit(c, e) == -1
    c[7] += 1
    assert lanes.audit(c, e) == 7


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    import torch.distributed as dist
    from datetime import timedelta

    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=timedelta(seconds=120))
    try:
        s = x2.SyntheticScene(CONFIG)
        ref = Reference(s)
        first, count = lanes.share(rank, world, SPP)
        rc, sums, odd, counts, _ = ref.render(first, count, threads=2)
        assert rc == 0
        assert lanes.audit(counts, lanes.expected_counts(len(counts), SPP, first, count)) == -1
        merged = lanes.merge_and_audit(sums, counts, SPP, odd=odd)
        result = {"ok": True}
        if rank == 0:
            np.savez(os.path.join(out_dir, "merged.npz"), sums=merged[0], counts=merged[1], odd=merged[2])
        # A share that lost one sample: the merged audit names the pixel.
        if rank == 1:
            counts = counts.copy()
            counts[1234] -= 1
        try:
            lanes.merge_and_audit(sums, counts, SPP)
            result["planted"] = None
        except x2.X2Error as e:
            result["planted"] = [e.code, str(e)]
        with open(os.path.join(out_dir, "rank%d.json" % rank), "w") as f:
            json.dump(result, f)
    finally:
        dist.destroy_process_group()


@pytest.mark.skipif(not have_reference(), reason="oracle/_ref not built")
def test_two_ranks_merge_to_the_whole_frame(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.start_processes(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True, start_method="spawn")
    got = np.load(tmp_path / "merged.npz")
    s = x2.SyntheticScene(CONFIG)
    rc, sums, odd, counts, _ = Reference(s).render(0, SPP)
    assert rc == 0
    assert np.array_equal(got["counts"], counts)
    assert np.array_equal(got["sums"], sums)
    assert np.array_equal(got["odd"], odd)
    r0 = json.load(open(tmp_path / "rank0.json"))
    r1 = json.load(open(tmp_path / "rank1.json"))
    assert r0["ok"] and r1["ok"]
    assert r1["planted"] is None  # the audit runs on rank 0 only
    assert r0["planted"][0] == x2.EAUDIT and "pixel 1234" in r0["planted"][1]
