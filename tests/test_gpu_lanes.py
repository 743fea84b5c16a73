"""GPU test of the multi-GPU film merge through the library (x2/lanes.py merge_and_audit_device): two ranks, each
rendering its share of a frame's samples with libx2 and summing the films in place on the device, give the whole
frame's film and pass the merged audit. Only one GPU is available here, so both ranks use cuda:0 and the reduce runs
over gloo (staged through the host); between GPUs the same calls run over NCCL. No kernel of one rank waits on the
other's."""
import multiprocessing as mp
import os
import socket
import tempfile
from datetime import timedelta

import numpy as np
import pytest

from oracle_lib import x2

pytestmark = pytest.mark.gpu

SPP = 5


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    import torch.distributed as dist

    import x2 as lib
    from x2 import lanes

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    with lib.Context(0) as ctx:
        s = lib.SyntheticScene(108)
        cfg = s.config
        cfg.spp = SPP
        scene = lib.Scene(ctx, s.desc, cfg)
        first, count = lanes.share(rank, world, SPP)
        scene.frame_begin(SPP)
        scene.render_frame_wavefront(first, count)
        lanes.merge_and_audit_device(scene, SPP)
        sums, counts = scene.film()
        np.savez(os.path.join(out_dir, "rank%d.npz" % rank), sums=sums, counts=counts)
        scene.free()
    dist.destroy_process_group()


def test_two_ranks_merge_on_device_to_the_whole_frame(ctx):
    s = x2.SyntheticScene(108)
    cfg = s.config
    cfg.spp = SPP
    scene = x2.Scene(ctx, s.desc, cfg)
    scene.frame_begin(SPP)
    scene.render_frame_wavefront(0, SPP)
    scene.wait()
    scene.audit()
    want, wc = scene.film()
    scene.free()
    world, port = 2, _free_port()
    spawn = mp.get_context("spawn")
    with tempfile.TemporaryDirectory() as out_dir:
        procs = [spawn.Process(target=_rank, args=(r, world, port, out_dir)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
        codes = [p.exitcode for p in procs]
        for p in procs:
            if p.is_alive():
                p.kill()
        assert codes == [0, 0], codes
        got = [np.load(os.path.join(out_dir, "rank%d.npz" % r)) for r in range(world)]
    for g in got:
        assert np.array_equal(g["counts"], wc)
        assert np.allclose(g["sums"], want, rtol=1e-12, atol=1e-12)
    assert np.array_equal(got[0]["sums"], got[1]["sums"])
