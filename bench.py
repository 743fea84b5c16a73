"""Benchmark of the path-sample hot path on B200: Msamples/s and Mrays/s of the plain megakernel on the 12.3M-triangle
scene (config 1: 1920x1080, 64 spp, 16 rect lights + environment, depth 12).

A step renders one whole frame (132,710,400 samples) through the lane API. `value` is device time of the render
launches (CUDA events on the library's stream, inputs resident in HBM, max over ranks); `e2e` is the same metric
through the public API with host buffers: chunk upload, render, film download and the sample-count audit every step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With N > 1 it runs under torchrun, one rank a GPU; each rank renders its own frame of distinct sample indices
(weak scaling) and the films are summed over NCCL at the end, as the reference adds its lanes' films.
`--impl reference` times the reference's own CPU integrator (oracle/_ref, compiled from the reference's sources) on
the host cores, on a bounded sample of the same frame.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "xpu2-foundation_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

WORKLOAD = "config 1: heightfield 64x64 tiles x 16x16 quads + 2000 level-4 icospheres (12,337,152 triangles), " \
           "16 rect lights + env 0.2, 1920x1080, 64 spp, max depth 12, plain megakernel"
METRIC = "Msamples/s (config 1, 1 frame = 1920x1080x64 samples a step)"
NODE_BYTES, TRI_BYTES, FILM_BYTES = 80, 48, 36


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) >= 9 for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def dist_setup(n):
    if n <= 1:
        return None, 0, 1, 0
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    rank, world, local = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"]), int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    return dist, rank, world, local


def max_over_ranks(dist, v, local):
    if dist is None:
        return v
    import torch

    t = torch.tensor([v], dtype=torch.float64, device=f"cuda:{local}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist, local):
    if dist is not None:
        import torch

        dist.barrier(device_ids=[local])
        torch.cuda.synchronize(local)


def cpu_baseline(synthetic, budget_s=15.0, impl_line=False):
    """The reference's CPU integrator (compiled from its sources) on all host cores, on a bounded sample of the frame:
    every k-th 8x8 tile at the frame's full spp, k chosen so the run takes about budget_s."""
    import oracle_lib

    if not oracle_lib.have_reference():
        return None, "oracle/_ref/libx2ref.so is not built"
    cfg = synthetic.config
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    ref = oracle_lib.Reference(synthetic)
    build_s = time.perf_counter() - t0
    tiles_x, tiles_y = (cfg.width + 7) // 8, (cfg.height + 7) // 8
    tiles = tiles_x * tiles_y
    probe = np.arange(0, tiles, max(1, tiles // (2 * threads)), dtype=np.uint32)[: 2 * threads]
    t0 = time.perf_counter()
    ref.render_tiles(probe, 0, 4, threads)
    per_tile = (time.perf_counter() - t0) / len(probe) * (cfg.spp / 4.0)
    want = max(threads, int(budget_s / max(per_tile, 1e-6) * threads))
    step = max(1, tiles // want)
    sample = np.arange(0, tiles, step, dtype=np.uint32)
    t0 = time.perf_counter()
    rc, samples, rays = ref.render_tiles(sample, 0, cfg.spp, threads)
    dt = time.perf_counter() - t0
    ref.close()
    value = samples / dt / 1e6
    return {"value": value, "unit": "Msamples/s", "cores": threads, "kind": "reference",
            "sample": f"{len(sample)} of {tiles} 8x8 tiles (every {step}th) x {cfg.spp} spp = {samples} samples of the same frame; "
                      f"reference integratePaths compiled from source (-O2 -ffp-contract=off), {threads} std::threads; "
                      f"CPU BVH build {build_s:.1f}s excluded",
            "mrays_per_s": float(rays[0] + rays[1] + rays[2]) / dt / 1e6, "seconds": dt, "rc": rc}, None


def run_reference(args):
    dist, rank, world, local = dist_setup(args.gpus)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    import x2

    s = x2.SyntheticScene(1)
    cfg = s.config
    vals, base = [], None
    for k in range(args.warmup + args.steps):
        base, why = cpu_baseline(s, budget_s=max(2.0, 60.0 / max(1, args.warmup + args.steps)))
        if base is None:
            print(json.dumps({"impl": "reference", "unavailable": why}))
            return
        if k >= args.warmup:
            vals.append(base["value"])
    value = statistics.median(vals)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Msamples/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": cfg.width * cfg.height * cfg.spp / (value * 1e6) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator, config 1)",
            "config": {"workload": WORKLOAD, "sample": base["sample"]},
            "cpu_baseline": {"value": value, "unit": "Msamples/s", "cores": base["cores"], "kind": "reference", "sample": base["sample"]},
            "e2e": {"value": value, "unit": "Msamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "mrays_per_s": base["mrays_per_s"]}
    print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


def traffic_from_profile():
    """The dominant kernel's DRAM bytes per launch from the committed ncu summary, when there is one."""
    p = os.path.join(ROOT, "profiles", "render_config1_traffic.json")
    try:
        with open(p) as f:
            return json.load(f)
    except Exception:
        return None


def run(args):
    dist, rank, world, local = dist_setup(args.gpus)
    import x2

    ctx = x2.Context(local)
    s = x2.SyntheticScene(1)
    cfg = s.config
    t0 = time.perf_counter()
    scene = x2.Scene(ctx, s.desc, cfg)
    info = scene.info()
    load_s = time.perf_counter() - t0
    samples_per_frame = cfg.width * cfg.height * cfg.spp
    first = rank * cfg.spp  # each rank its own sample indices: distinct samples of the same pixels
    tiles = ((cfg.width + 7) // 8) * ((cfg.height + 7) // 8)

    # Counting run (untimed): node visits and triangle tests of one frame, for the algorithmic bytes.
    scene.count_traversal(True)
    scene.frame_begin(cfg.spp)
    scene.render_frame(first, cfg.spp)
    scene.wait()
    tc = scene.traversal_counts()
    scene.count_traversal(False)
    scene.reset_counters()

    # Device-timed steps: inputs resident, one render launch a step (the film cleared between, not timed).
    for _ in range(args.warmup):
        scene.frame_begin(cfg.spp)
        scene.render_frame(first, cfg.spp)
        scene.wait()
    scene.reset_counters()
    clocks = Clocks(local)
    barrier(dist, local)
    clocks.start()
    ms = []
    for _ in range(args.steps):
        scene.frame_begin(cfg.spp)
        scene.render_frame(first, cfg.spp)
        c = scene.wait()
        ms.append(c.milliseconds)
    barrier(dist, local)
    clk = clocks.stop()
    counters = scene.counters()
    scene.audit()
    total_ms = max_over_ranks(dist, float(sum(ms)), local)
    ms_per_step = total_ms / args.steps
    value = world * samples_per_frame * args.steps / (total_ms / 1e3) / 1e6
    rays = counters["trace"] + counters["shadow_nee"] + counters["shadow_bsdf"]
    mrays = world * rays / (sum(ms) / 1e3) / 1e6

    # End to end through the public API: chunks up, render, film down, audit, every step.
    film_bytes = cfg.width * cfg.height * (4 * 8 + 4)
    chunk_bytes = tiles * 16
    barrier(dist, local)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        scene.frame_begin(cfg.spp)
        scene.render_frame(first, cfg.spp)
        sums, counts = scene.film()
        scene.audit()
    e2e_s = max_over_ranks(dist, time.perf_counter() - t0, local)
    e2e_value = world * samples_per_frame * args.steps / e2e_s / 1e6

    # Multi-GPU: the lanes' films summed over NCCL at frame end, then the audit of the merged counts.
    if dist is not None:
        import torch

        ts = torch.from_numpy(sums).cuda(local)
        tc_ = torch.from_numpy(counts.astype(np.int64)).cuda(local)
        dist.reduce(ts, 0)
        dist.reduce(tc_, 0)
        if rank == 0 and not bool((tc_ == world * cfg.spp).all()):
            raise RuntimeError("merged sample-count audit failed")

    hbm, peak_kind = peaks()
    alg_bytes = tc["nodes"] * NODE_BYTES + tc["triangles"] * TRI_BYTES + samples_per_frame * FILM_BYTES
    achieved = alg_bytes / (ms_per_step / 1e3) / 1e9
    prof = traffic_from_profile()
    if rank == 0:
        base, why = cpu_baseline(s) if world == 1 else (None, "rank 0 at N=1 only")
        line = {
            "metric": METRIC, "value": value, "unit": "Msamples/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generator, config 1; no dataset)",
            "config": {"workload": WORKLOAD, "triangles": s.desc.triangle_count, "samples_per_step": samples_per_frame * world,
                       "l2": "inputs larger than L2 (BVH %.0f MB + triangles %.0f MB > 126 MB)" % (info["bvh_bytes"] / 1e6, info["triangle_bytes"] / 1e6),
                       "bvh_build_ms": info["build_ms"], "scene_load_s": load_s, "parallelism": f"{world} GPU(s), replicated scene, "
                       "distinct sample indices a rank"},
            "mrays_per_s": mrays,
            "rays_per_sample": {"trace": counters["trace"] / (samples_per_frame * args.steps),
                                "shadow_nee": counters["shadow_nee"] / (samples_per_frame * args.steps),
                                "shadow_bsdf": counters["shadow_bsdf"] / (samples_per_frame * args.steps),
                                "held": counters["held"] / (samples_per_frame * args.steps)},
            "e2e": {"value": e2e_value, "unit": "Msamples/s", "h2d_bytes_per_step": chunk_bytes, "d2h_bytes_per_step": film_bytes},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": (prof or {}).get("dram_bytes_per_launch"), "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "per_launch": {"rays": tc["rays"], "node_visits": tc["nodes"], "triangle_tests": tc["triangles"],
                                        "node_bytes": NODE_BYTES, "triangle_bytes": TRI_BYTES, "film_bytes_per_sample": FILM_BYTES}},
            "cpu_baseline": base if base else {"value": None, "unavailable": why},
            "clocks": clk, "gpu_launches": args.steps,
            "errors": counters["errors"], "stack_overflows": counters["stack_overflows"],
        }
        print(json.dumps(line))
    scene.free()
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="x2", choices=["x2", "reference"])
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run(args)


if __name__ == "__main__":
    main()
