"""Benchmark of the path-sample hot path on B200: Msamples/s and Mrays/s on the 12.3M-triangle scene (config 1:
1920x1080, 64 spp, 16 rect lights + environment, depth 12), wavefront form against the plain megakernel.

A step renders one whole frame (132,710,400 samples) through the lane API in the wavefront form. `value` is the
device time of those launches (CUDA events on the library's stream around the whole launch, film reduction
included; inputs resident in HBM; max over ranks). The plain megakernel renders the same frame (the same samples, so
the same image and RMSE) and is reported beside it. `e2e` is the headline through the public API with host buffers:
chunk upload, render, film download and the sample-count audit every step.

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
           "16 rect lights + env 0.2, 1920x1080, 64 spp, max depth 12"
METRIC = "Msamples/s (config 1, 1 frame = 1920x1080x64 samples a step)"
NODE_BYTES, TRI_BYTES, FILM_BYTES = 80, 48, 36
# Per ray record bytes the traversal kernels read and write besides the BVH: extend reads a 32-byte ray and writes
# an 8-byte hit; shadow reads a 32-byte record and writes a 1-byte flag.
EXTEND_RAY_BYTES, SHADOW_RAY_BYTES = 40, 33


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
        rows = [r for r in self.rows if len(r) >= 9]
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


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


def cpu_baseline(synthetic, budget_s=15.0):
    """The reference's CPU integrator (compiled from its sources) on all host cores, on a bounded sample of the frame:
    seeded random 8x8 tiles at the frame's full spp, as many as take about budget_s."""
    import oracle_lib

    if not oracle_lib.have_reference():
        return None, "oracle/_ref/libx2ref.so is not built"
    cfg = synthetic.config
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    ref = oracle_lib.Reference(synthetic)
    build_s = time.perf_counter() - t0
    tiles = ((cfg.width + 7) // 8) * ((cfg.height + 7) // 8)
    order = np.random.default_rng(17).permutation(tiles).astype(np.uint32)
    probe = order[:threads]
    t0 = time.perf_counter()
    ref.render_tiles(probe, 0, cfg.spp, threads)
    per_batch = time.perf_counter() - t0  # one tile a thread at full spp
    batches = max(1, int(budget_s / max(per_batch, 1e-3)))
    sample = order[threads: threads + min(tiles - threads, batches * threads)]
    t0 = time.perf_counter()
    rc, samples, rays = ref.render_tiles(sample, 0, cfg.spp, threads)
    dt = time.perf_counter() - t0
    ref.close()
    value = samples / dt / 1e6
    return {"value": value, "unit": "Msamples/s", "cores": threads, "kind": "reference",
            "sample": f"{len(sample)} of {tiles} seeded-random 8x8 tiles x {cfg.spp} spp = {samples} samples of the same frame; "
                      f"reference integratePaths compiled from source (-O2 -ffp-contract=off), {threads} std::threads; "
                      f"CPU BVH build {build_s:.1f}s excluded",
            "mrays_per_s": float(rays[0] + rays[1] + rays[2]) / dt / 1e6, "seconds": dt, "rc": rc}, None


def run_reference(args):
    """The reference arm: the reference's own CPU integrator (integratePaths compiled from its sources into
    oracle/_ref/libx2ref.so, with the seeded scene generator compiled in, so libx2 is never loaded here) on all host
    cores. The scene and its CPU BVH are built once; each step renders a bounded sample of the config-1 frame — the
    next `tiles_per_step` 8x8 tiles of a seeded permutation of the frame's tiles, at the frame's full spp — and is
    timed on its own, so ms_per_step is the time a step took."""
    dist, rank, world, local = dist_setup(args.gpus)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    import oracle_lib

    if not oracle_lib.have_reference():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libx2ref.so is not built"}))
        return
    from x2 import SyntheticScene

    s = SyntheticScene(1, generator=oracle_lib.generator())
    cfg = s.config
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    ref = oracle_lib.Reference(s)
    build_s = time.perf_counter() - t0
    tiles = ((cfg.width + 7) // 8) * ((cfg.height + 7) // 8)
    order = np.random.default_rng(17).permutation(tiles).astype(np.uint32)
    # Calibrate: one tile a thread at full spp, then as many tiles a step as take about step_s.
    step_s = min(8.0, max(1.0, 150.0 / max(1, args.warmup + args.steps)))
    t0 = time.perf_counter()
    ref.render_tiles(order[:threads], 0, cfg.spp, threads)
    per_batch = time.perf_counter() - t0
    per_step = max(threads, min(tiles, int(step_s / max(per_batch, 1e-3)) * threads))
    times, samples_timed, rays_timed, cursor = [], 0, 0, threads
    for k in range(args.warmup + args.steps):
        sel = order[np.arange(cursor, cursor + per_step) % tiles]
        cursor += per_step
        t0 = time.perf_counter()
        rc, n, rays = ref.render_tiles(sel, 0, cfg.spp, threads)
        dt = time.perf_counter() - t0
        if rc != 0:
            print(json.dumps({"impl": "reference", "unavailable": f"the reference integrator returned {rc}"}))
            return
        if k >= args.warmup:
            times.append(dt)
            samples_timed += n
            rays_timed += int(rays[0] + rays[1] + rays[2])
    ref.close()
    total_s = sum(times)
    value = samples_timed / total_s / 1e6
    sample = (f"{per_step} of {tiles} seeded-random 8x8 tiles a step (the next ones each step) x {cfg.spp} spp = "
              f"{per_step * 64 * cfg.spp} samples of the config-1 frame; reference integratePaths compiled from source "
              f"(-O2 -ffp-contract=off), {threads} std::threads; scene generation and CPU BVH build ({build_s:.1f} s) once, "
              f"outside the steps")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "Msamples/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_s / len(times) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator, config 1)",
            "config": {"workload": WORKLOAD + f"; a step = {per_step} of its {tiles} tiles", "tiles_per_step": per_step,
                       "samples_per_step": per_step * 64 * cfg.spp, "sample": sample},
            "cpu_baseline": {"value": value, "unit": "Msamples/s", "cores": threads, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": "Msamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "mrays_per_s": rays_timed / total_s / 1e6}
    print(json.dumps(line))
    s.free()
    if dist:
        dist.destroy_process_group()


def traffic_from_profile():
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary, when there is one."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def kernels_per_iteration(spec):
    """Kernels a wavefront iteration launches: queue reset, logic, extend, the per-lobe sort (lobe_queues), shade (three
    kernels with shade_split, else one), the two light kernels (light_split), shadow and the drain check."""
    shape = dict(kv.split("=") for kv in spec.split(",")) if spec else {}
    lobe = int(shape.get("lobe_queues", 1))
    split = int(shape.get("shade_split", 1)) and lobe
    lights = 2 if split and int(shape.get("light_split", 1)) else 0
    return 5 + lobe + (3 if split else 1) + lights


def simt_summary(tc):
    """Lane use of the persistent traversal kernels from a counting launch, by ray kind: live lanes a warp step, lanes a
    step that ran the node visit, lanes a triangle-test iteration (each of 32), node visits and triangle tests a ray."""
    out = {}
    for kind, name in (("closest", "extend"), ("any", "shadow")):
        t = tc[kind]
        l = t["lanes"]
        if not l["steps"] or not t["rays"]:
            continue
        out[name] = {"live_lanes": l["live_lanes"] / l["steps"],
                     "node_lanes": l["node_lanes"] / max(1, l["node_steps"]),
                     "tri_lanes": l["tri_lanes"] / max(1, l["tri_steps"]),
                     "node_steps_per_step": l["node_steps"] / l["steps"],
                     "tri_iterations_per_step": l["tri_steps"] / l["steps"],
                     "nodes_per_ray": t["nodes"] / t["rays"], "triangles_per_ray": t["triangles"] / t["rays"]}
    return out


def apply_shape(scene, spec):
    """x2_wavefront_tune with the fields named in `spec` ("k=v,k=v"), the others at their defaults."""
    if spec:
        scene.wavefront_tune(**{k: int(v) for k, v in (kv.split("=") for kv in spec.split(","))})


def frame(scene, cfg, first, wavefront):
    scene.frame_begin(cfg.spp)
    if wavefront:
        scene.render_frame_wavefront(first, cfg.spp)
    else:
        scene.render_frame(first, cfg.spp)
    return scene.wait()


def run(args):
    dist, rank, world, local = dist_setup(args.gpus)
    import torch
    import x2

    ctx = x2.Context(local)
    s = x2.SyntheticScene(1)
    cfg = s.config
    t0 = time.perf_counter()
    scene = x2.Scene(ctx, s.desc, cfg)
    apply_shape(scene, args.shape)
    info = scene.info()
    load_s = time.perf_counter() - t0
    samples_per_frame = cfg.width * cfg.height * cfg.spp
    first = rank * cfg.spp  # each rank its own sample indices: distinct samples of the same pixels
    tiles = ((cfg.width + 7) // 8) * ((cfg.height + 7) // 8)

    # Untimed: node visits and triangle tests of one frame (counting mode), and the wavefront's per-kernel times.
    scene.count_traversal(True)
    frame(scene, cfg, first, True)
    tc = scene.traversal_counts()
    scene.count_traversal(False)
    scene.wavefront_timing(True)
    frame(scene, cfg, first, True)
    kms = scene.wavefront_timing(False)
    scene.reset_counters()
    # The cache levels' read bandwidth on this GPU, measured here (untimed): the ceilings of the traversal kernels'
    # node and triangle fetches, which hit L1 and L2 far more than HBM.
    l1_gbs = ctx.probe_bandwidth(1, 96 << 10, 200)
    l2_gbs = ctx.probe_bandwidth(2, 32 << 20, 20)

    # Device-timed wavefront frames.
    for _ in range(args.warmup):
        frame(scene, cfg, first, True)
    scene.reset_counters()
    clocks = Clocks(local)
    barrier(dist, local)
    clocks.start()
    ms = []
    for _ in range(args.steps):
        ms.append(frame(scene, cfg, first, True).milliseconds)
    barrier(dist, local)
    clk = clocks.stop()
    counters = scene.counters()
    winfo = scene.wavefront_info()
    scene.audit()
    total_ms = max_over_ranks(dist, float(sum(ms)), local)
    ms_per_step = total_ms / args.steps
    value = world * samples_per_frame * args.steps / (total_ms / 1e3) / 1e6
    rays = counters["trace"] + counters["shadow_nee"] + counters["shadow_bsdf"]
    mrays = world * rays / (total_ms / 1e3) / 1e6

    # The plain megakernel on the same frame (the same samples: same image, same RMSE).
    plain = None
    if not args.skip_plain:
        frame(scene, cfg, first, False)
        pms = [frame(scene, cfg, first, False).milliseconds for _ in range(args.plain_steps)]
        pmax = max_over_ranks(dist, float(sum(pms)), local) / len(pms)
        plain = {"value": world * samples_per_frame / (pmax / 1e3) / 1e6, "unit": "Msamples/s", "ms_per_step": pmax,
                 "steps": len(pms), "warmup": 1, "mrays_per_s": world * rays / args.steps / (pmax / 1e3) / 1e6}

    # End to end through the public API: chunks up, render, film down, audit, every step. The film comes down into
    # pinned host arrays the caller keeps across frames (Scene.film's `out`).
    film_bytes = cfg.width * cfg.height * (4 * 8 + 4)
    chunk_bytes = tiles * 16
    pixels = cfg.width * cfg.height
    film_out = (torch.empty((pixels, 4), dtype=torch.float64, pin_memory=True).numpy(),
                torch.empty(pixels, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32))
    barrier(dist, local)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        scene.frame_begin(cfg.spp)
        scene.render_frame_wavefront(first, cfg.spp)
        sums, counts = scene.film(out=film_out)
        scene.audit()
    e2e_s = max_over_ranks(dist, time.perf_counter() - t0, local)
    e2e_value = world * samples_per_frame * args.steps / e2e_s / 1e6

    # Both forms again with the kernels built with contraction (-fmad=true, as the reference's production GPU lane is
    # built; the parity build above is -fmad=false): one frame each, in a process of its own, at N=1 only.
    fmad = forms_with("libx2fmad.so") if world == 1 and not args.skip_plain else None

    # Multi-GPU: the lanes' films summed in place on the devices over NCCL at frame end, then the merged counts'
    # audit on the device.
    if dist is not None:
        from x2 import lanes

        lanes.merge_and_audit_device(scene, world * cfg.spp)

    # Roofline of the dominant wavefront kernel. Its algorithmic bytes (BVH nodes and triangles its rays visit, and
    # its ray records, counted in the counting frame) over its time in the per-kernel timed frame, against the cache
    # level that serves them and against HBM; and its instruction issue, the limit it runs against (warp instructions
    # a ray from the committed ncu capture, times this frame's rays, over the same time, against four issues a cycle
    # a SM at the clock sampled during the timed frames).
    hbm, peak_kind = peaks()
    per_kernel = {
        "extend": (tc["closest"]["nodes"] * NODE_BYTES + tc["closest"]["triangles"] * TRI_BYTES + tc["closest"]["rays"] * EXTEND_RAY_BYTES,
                   kms["extend"]),
        "shadow": (tc["any"]["nodes"] * NODE_BYTES + tc["any"]["triangles"] * TRI_BYTES + tc["any"]["rays"] * SHADOW_RAY_BYTES, kms["shadow"]),
    }
    dominant = max(kms, key=lambda k: kms[k])
    dom = dominant if dominant in per_kernel else max(per_kernel, key=lambda k: per_kernel[k][1])
    alg_bytes, dom_ms = per_kernel[dom]
    launches_per_frame = winfo["iterations"]
    achieved = alg_bytes / (dom_ms / 1e3) / 1e9 if dom_ms > 0 else 0.0
    # DRAM traffic a launch: the ncu capture's DRAM bytes a ray (profiles/traffic.json) times this frame's rays of
    # that kind a launch; compare with the algorithmic bytes a launch.
    prof = traffic_from_profile().get(dom, {})
    dom_rays = tc["any" if dom == "shadow" else "closest"]["rays"]
    traffic = prof["dram_bytes_per_ray"] * dom_rays / launches_per_frame if "dram_bytes_per_ray" in prof and launches_per_frame else None
    secs = dom_ms / 1e3 if dom_ms > 0 else float("inf")

    def level(per_ray_key, peak):
        if per_ray_key not in prof:
            return None
        got = prof[per_ray_key] * dom_rays / secs / 1e9
        return {"measured_bytes_per_ray": prof[per_ray_key], "achieved": got, "peak": peak, "frac": got / peak if peak else None}

    sm_mhz = clk.get("sm_mhz") or 1965.0
    import torch

    sms = torch.cuda.get_device_properties(local).multi_processor_count
    issue_peak = 4 * sms * sm_mhz * 1e6 / 1e9  # warp instructions a second (Ginst/s): four schedulers a SM
    issue = None
    if "warp_inst_per_ray" in prof:
        got = prof["warp_inst_per_ray"] * dom_rays / secs / 1e9
        issue = {"bound": "issue", "unit": "Ginst/s", "achieved": got, "peak": issue_peak, "frac": got / issue_peak,
                 "warp_inst_per_ray": prof["warp_inst_per_ray"], "lanes_active": prof.get("lanes_active")}
    if rank == 0:
        base, why = cpu_baseline(s) if world == 1 else (None, "rank 0 at N=1 only")
        line = {
            "metric": METRIC, "value": value, "unit": "Msamples/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generator, config 1; no dataset)",
            "config": {"workload": WORKLOAD + ", wavefront form", "triangles": s.desc.triangle_count, "samples_per_step": samples_per_frame * world,
                       "wavefront_shape": args.shape or "library defaults",
                       "l2": "inputs larger than L2 (BVH %.0f MB + triangles %.0f MB > 126 MB)" % (info["bvh_bytes"] / 1e6, info["triangle_bytes"] / 1e6),
                       "bvh_build_ms": info["build_ms"], "scene_load_s": load_s, "paths_in_flight": winfo["paths"],
                       "parallelism": f"{world} GPU(s), replicated scene, distinct sample indices a rank"},
            "mrays_per_s": mrays,
            "rays_per_sample": {k: counters[c] / (samples_per_frame * args.steps)
                                for k, c in (("trace", "trace"), ("shadow_nee", "shadow_nee"), ("shadow_bsdf", "shadow_bsdf"), ("held", "held"))},
            "plain_megakernel": plain,
            "wavefront_over_plain": (value / plain["value"]) if plain else None,
            "fmad_true": fmad,
            "e2e": {"value": e2e_value, "unit": "Msamples/s", "h2d_bytes_per_step": chunk_bytes, "d2h_bytes_per_step": film_bytes},
            "roofline": {"bound": "issue", "kernel": "wf" + dom.capitalize(), "unit": "Ginst/s",
                         "achieved": issue["achieved"] if issue else None, "peak": issue_peak,
                         "frac": issue["frac"] if issue else None, "traffic": traffic,
                         "peak_kind": "4 warp instructions a cycle a SM x %d SMs x the SM clock sampled during the timed frames" % sms,
                         "issue": issue,
                         "algorithmic": {
                             "unit": "GB/s", "achieved": achieved, "bytes_per_launch": alg_bytes / launches_per_frame if launches_per_frame else None,
                             "l1": {"peak": l1_gbs, "frac": achieved / l1_gbs, "requested": level("l1_bytes_per_ray", l1_gbs),
                                    "peak_kind": "measured in this run (x2_probe_bandwidth level 1: every SM re-reading 96 KB)"},
                             "l2": {"peak": l2_gbs, "frac": achieved / l2_gbs, "read_from_l2": level("l2_read_bytes_per_ray", l2_gbs),
                                    "peak_kind": "measured in this run (x2_probe_bandwidth level 2: a 32 MB buffer swept by the grid)"},
                             "hbm": {"peak": hbm, "frac": achieved / hbm, "dram": level("dram_bytes_per_ray", hbm), "peak_kind": peak_kind}},
                         "algorithmic_bytes_per_launch": alg_bytes / launches_per_frame if launches_per_frame else None,
                         "traffic_source": prof.get("source"),
                         "algorithmic_bytes_per_frame": alg_bytes, "kernel_ms_per_frame": dom_ms,
                         "kernel_ms_by_kind": kms, "traversal": tc, "simt": simt_summary(tc),
                         "bytes": {"node": NODE_BYTES, "triangle": TRI_BYTES, "extend_ray": EXTEND_RAY_BYTES, "shadow_ray": SHADOW_RAY_BYTES}},
            "cpu_baseline": base if base else {"value": None, "unavailable": why},
            "clocks": clk, "gpu_launches": (launches_per_frame * kernels_per_iteration(args.shape) + 1) * args.steps,
            "errors": counters["errors"], "stack_overflows": counters["stack_overflows"],
        }
        print(json.dumps(line))
    scene.free()
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


def probe_batch(args):
    """Config 2: its 48 requests (config-1-style scenes of 0.1M..2M triangles, 128^2..1024^2, 4..256 spp, depth 4..32,
    frame seed 1 + r) rendered in one batched wavefront launch, `--probe-tiles` of them (all by default), after one
    untimed warm-up batch; every film audited. Prints the aggregate Msamples/s."""
    import x2

    ctx = x2.Context(0)
    count = min(48, args.probe_tiles) if args.probe_tiles else 48
    t0 = time.perf_counter()
    scenes, triangles = [], 0
    for r in range(count):
        s = x2.SyntheticScene(200 + r)
        scenes.append((s.config, x2.Scene(ctx, s.desc, s.config)))
        triangles += s.desc.triangle_count
        s.free()
    load_s = time.perf_counter() - t0
    requests = [(sc, 0, cfg.spp) for cfg, sc in scenes]
    samples = sum(cfg.width * cfg.height * cfg.spp for cfg, _ in scenes)
    ctx.render_batch(requests)
    runs = [ctx.render_batch(requests) for _ in range(max(1, args.steps))]
    for _, sc in scenes:
        sc.audit()
    ms = statistics.median(c.milliseconds for c in runs)
    print(json.dumps({"probe": "batch", "requests": count, "samples": samples, "triangles": triangles, "ms": ms,
                      "msamples_per_s": samples / ms / 1e3, "errors": int(sum(c.errors for c in runs)), "load_s": load_s,
                      "shape": x2.wavefront_shape_defaults().as_dict()}))
    for _, sc in scenes:
        sc.free()
    ctx.close()


def probe_volume(args):
    """Config 3 (the participating medium: a 256^3 grid in the closed box, a rect light and a sun; 512x512, 256 spp,
    depth 64): `--probe-tiles` evenly spaced 8x8 tiles (all 4096 by default when the flag is left at its 592 default
    is not wanted, pass 4096) at full spp in the wavefront form (`--probe-timed`: without its graph, each kernel
    timed), then the plain megakernel on the same tiles; the films compared and audited. Prints Msamples/s of each
    form."""
    import x2

    ctx = x2.Context(0)
    s = x2.SyntheticScene(3)
    cfg = s.config
    scene = x2.Scene(ctx, s.desc, cfg)
    apply_shape(scene, args.shape)
    tiles = ((cfg.width + 7) // 8) * ((cfg.height + 7) // 8)
    sel = np.linspace(0, tiles - 1, min(tiles, args.probe_tiles)).astype(np.uint32)
    chunks = np.zeros(len(sel), x2.CHUNK_DTYPE)
    chunks["tile"], chunks["first"], chunks["count"] = sel, 0, cfg.spp
    n = len(sel) * 64 * cfg.spp
    out = {"probe": "volume", "tiles": len(sel), "samples": n, "grid": "256^3", "spp": cfg.spp, "shape": args.shape}
    films = {}
    for form in ("wavefront", "plain"):
        scene.frame_begin(cfg.spp)
        if form == "wavefront":
            scene.wavefront_timing(args.probe_timed)  # --probe-timed: no graph, each kernel's launches visible
        (scene.launch_wavefront if form == "wavefront" else scene.launch)(chunks)
        c = scene.wait()
        films[form] = scene.film()
        out[form] = {"ms": c.milliseconds, "msamples_per_s": n / c.milliseconds / 1e3, "errors": c.errors}
        if form == "wavefront" and args.probe_timed:
            out["kernel_ms"] = scene.wavefront_timing(None)
    out["films_close"] = bool(np.allclose(films["wavefront"][0], films["plain"][0], rtol=1e-9, atol=1e-9) and
                              np.array_equal(films["wavefront"][1], films["plain"][1]))
    out["counters"] = scene.counters()
    print(json.dumps(out))
    scene.free()
    ctx.close()


def probe_forms(args):
    """One config-1 frame in each form (wavefront, then the plain megakernel), each after a warm-up frame, with the
    library this process loaded (X2_LIBRARY: the contracted build libx2fmad.so when bench.py asks for it). Prints the
    Msamples/s of each."""
    import x2

    ctx = x2.Context(0)
    s = x2.SyntheticScene(1)
    cfg = s.config
    scene = x2.Scene(ctx, s.desc, cfg)
    n = cfg.width * cfg.height * cfg.spp
    out = {"probe": "forms", "library": os.path.basename(x2.LIBRARY)}
    for name, wave in (("wavefront", True), ("plain", False)):
        frame(scene, cfg, 0, wave)
        ms = frame(scene, cfg, 0, wave).milliseconds
        out[name] = {"ms": ms, "msamples_per_s": n / ms / 1e3}
    print(json.dumps(out))
    scene.free()
    ctx.close()


def forms_with(library):
    """probe_forms in a process of its own that loads `library` (the x2 module loads one library a process)."""
    env = dict(os.environ, X2_LIBRARY=os.path.join(ROOT, "xpu2-foundation_b200", "x2", library))
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--probe", "forms"], capture_output=True, text=True, env=env, timeout=900)
    for line in r.stdout.splitlines():
        if line.startswith("{"):
            return json.loads(line)
    return {"unavailable": (r.stderr or r.stdout)[-300:]}


def probe_estimators(args):
    """Config 3 (the 256^3 medium): the reference's decoupled march against delta/ratio tracking over 32^3 majorant
    grids (x2_config.volume_estimator 1), each rendering the RMSE fixture's tiles (tests/golden/rmse_c3.npz) in the
    wavefront form: at the configuration's 256 spp, then tracking at the spp that takes the march's time; each image's
    RMSE against the converged reference (16,384 spp of the march, FP64 film). Then `--probe-tiles` evenly spaced tiles
    of the frame at 256 spp in each form for throughput."""
    import rmse_lib
    import x2

    ctx = x2.Context(0)
    f = np.load(os.path.join(ROOT, "tests", "golden", "rmse_c3.npz"))
    tiles, live, ref = f["tiles"], f["live"], f["ref"].astype(np.float64)
    out = {"probe": "estimators", "config": 3, "fixture_tiles": int(len(tiles)), "fixture_pixels": int(live.sum())}
    scenes = {}
    for name, est in (("march", 0), ("tracking", 1)):
        s = x2.SyntheticScene(3)
        s.config.volume_estimator = est
        scenes[name] = (s, x2.Scene(ctx, s.desc, s.config))
    spp = int(f["spp"])
    for name, (s, scene) in scenes.items():
        rmse_lib.render_tiles(scene, tiles, spp, True)  # warm-up
        img, ms = rmse_lib.render_tiles(scene, tiles, spp, True)
        out[name] = {"spp": spp, "ms": ms, "rmse": rmse_lib.rmse(img, ref, live), "mean": float(img[live].mean())}
    out["ref_mean"] = float(ref[live].mean())
    equal = max(1, int(spp * out["march"]["ms"] / out["tracking"]["ms"]))
    s, scene = scenes["tracking"]
    img, ms = rmse_lib.render_tiles(scene, tiles, equal, True)
    out["tracking_equal_time"] = {"spp": equal, "ms": ms, "rmse": rmse_lib.rmse(img, ref, live)}
    cfg = scenes["march"][0].config
    all_tiles = ((cfg.width + 7) // 8) * ((cfg.height + 7) // 8)
    sel = np.linspace(0, all_tiles - 1, min(all_tiles, args.probe_tiles)).astype(np.uint32)
    for name, (s, scene) in scenes.items():
        chunks = np.zeros(len(sel), x2.CHUNK_DTYPE)
        chunks["tile"], chunks["first"], chunks["count"] = sel, 0, spp
        scene.frame_begin(spp)
        scene.launch_wavefront(chunks)
        c = scene.wait()
        out[name]["throughput"] = {"tiles": len(sel), "msamples_per_s": len(sel) * 64 * spp / c.milliseconds / 1e3, "ms": c.milliseconds}
    print(json.dumps(out))
    for s, scene in scenes.values():
        scene.free()
    ctx.close()


def probe_adjoint(args):
    """Config 4 (about 250k triangles: a heightfield under a 1024x1024 albedo texture and 64 icospheres of 64
    materials; 512x512): the primal frame at 32 spp (wavefront and plain) and the
    adjoint of an L2 image loss at 16 spp (samples 32..47) in both forms (x2_adjoint: wavefront; x2_adjoint_plain:
    one thread a sample), each timed after a warm-up; Msamples/s of each and the adjoint's throughput over the
    primal's."""
    import torch
    import x2

    ctx = x2.Context(0)
    s = x2.SyntheticScene(4)
    cfg = s.config
    scene = x2.Scene(ctx, s.desc, cfg)
    pixels = cfg.width * cfg.height
    out = {"probe": "adjoint", "triangles": s.desc.triangle_count, "materials": s.desc.material_count, "primal_spp": 32,
           "adjoint_spp": 16}
    for form in ("wavefront",) if args.adjoint_only else ("wavefront", "plain"):
        for k in range(1 if args.adjoint_only else 2):
            scene.frame_begin(32)
            (scene.render_frame_wavefront if form == "wavefront" else scene.render_frame)(0, 32)
            c = scene.wait()
        out[form] = {"ms": c.milliseconds, "msamples_per_s": pixels * 32 / c.milliseconds / 1e3}
    sums, counts = scene.film()
    image = sums[:, :3] / counts[:, None]
    if args.adjoint_only:
        # One wavefront adjoint launch, for a profiler.
        ga = torch.zeros((s.desc.material_count, 3), dtype=torch.float64, device="cuda:0")
        gr = torch.zeros((s.desc.light_count, 3), dtype=torch.float64, device="cuda:0")
        gg = torch.zeros(s.desc.material_count, dtype=torch.float64, device="cuda:0")
        dl = torch.from_numpy(image.astype(np.float32)).to("cuda:0")
        scene.adjoint(32, 16, dl.data_ptr(), ga.data_ptr(), gr.data_ptr(), gg.data_ptr())
        torch.cuda.synchronize()
        print(json.dumps({"probe": "adjoint", "adjoint_only": True, "grad_norms": [float(ga.norm()), float(gr.norm()), float(gg.norm())]}))
        scene.free()
        ctx.close()
        return
    dev = torch.device("cuda", 0)
    dl = torch.from_numpy((2.0 * (image - 0.5 * image)).astype(np.float32)).to(dev)
    ga = torch.zeros((s.desc.material_count, 3), dtype=torch.float64, device=dev)
    gr = torch.zeros((s.desc.light_count, 3), dtype=torch.float64, device=dev)
    gg = torch.zeros(s.desc.material_count, dtype=torch.float64, device=dev)
    tex = s.texture(0)
    gt = torch.zeros((tex.shape[0] * tex.shape[1], 3), dtype=torch.float64, device=dev)
    out["texture"] = list(tex.shape)
    for name, plain in (("adjoint", False), ("adjoint_plain", True)):
        scene.adjoint(32, 16, dl.data_ptr(), ga.data_ptr(), gr.data_ptr(), gg.data_ptr(), plain=plain, d_texture_grad=gt.data_ptr())
        torch.cuda.synchronize()
        ga.zero_(), gr.zero_(), gg.zero_(), gt.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        scene.adjoint(32, 16, dl.data_ptr(), ga.data_ptr(), gr.data_ptr(), gg.data_ptr(), plain=plain, d_texture_grad=gt.data_ptr())
        adj_s = time.perf_counter() - t0  # x2_adjoint waits for its launches: host time brackets them
        out[name] = {"ms": adj_s * 1e3, "msamples_per_s": pixels * 16 / adj_s / 1e6,
                     "grad_norms": {"albedo": float(ga.norm()), "radiance": float(gr.norm()), "roughness": float(gg.norm()),
                                    "texels": float(gt.norm())}}
    out["adjoint_over_primal"] = out["adjoint"]["msamples_per_s"] / out["wavefront"]["msamples_per_s"]
    out["adjoint_plain_over_plain"] = out["adjoint_plain"]["msamples_per_s"] / out["plain"]["msamples_per_s"]
    print(json.dumps(out))
    scene.free()
    ctx.close()


def probe_rmse(args):
    """Image RMSE of both forms against the reference's converged renders (16,384 spp, FP64 film) of seeded tiles of
    every configuration with a fixture (tests/golden/rmse_c*.npz); one JSON line a fixture."""
    import rmse_lib
    import x2

    ctx = x2.Context(0)
    for path in rmse_lib.fixtures():
        print(json.dumps(dict(probe="rmse", **rmse_lib.measure(ctx, path))), flush=True)
    ctx.close()


def probe_adaptive(args):
    """An adaptive frame of config 0 (the closed box, 256x256; MoonRay's schedule up to 256 samples a pixel, passes from
    4 samples on adaptive, target error 5e-4): its passes, samples and time; then the image RMSE of its fixture tiles
    against the converged reference (tests/golden/rmse_c0.npz) beside a uniform frame's of about the same samples, and
    the same frame by cellular generations."""
    import rmse_lib
    import x2

    ctx = x2.Context(0)
    s = x2.SyntheticScene(0)
    cfg = s.config
    scene = x2.Scene(ctx, s.desc, cfg)
    scene.render_adaptive(4, 256, 5e-4)  # warm-up
    result = scene.render_adaptive(4, 256, 5e-4)
    sums, counts = scene.film()
    f = np.load(os.path.join(ROOT, "tests", "golden", "rmse_c0.npz"))
    px = rmse_lib.tile_pixels(f["tiles"], cfg.width, cfg.height)
    live = f["live"]
    ref = f["ref"].astype(np.float64)
    img = np.zeros(px.shape + (3,))
    img[live] = sums[px[live], :3] / counts[px[live], None]
    mean_spp = result["samples"] / (cfg.width * cfg.height)
    spp = max(1, int(round(mean_spp)))
    scene.frame_begin(spp)
    scene.render_frame_wavefront(0, spp)
    c = scene.wait()
    usums, ucounts = scene.film()
    uimg = np.zeros(px.shape + (3,))
    uimg[live] = usums[px[live], :3] / ucounts[px[live], None]
    scene.render_adaptive(4, 256, 5e-4, cellular=True)  # warm-up
    cell = scene.render_adaptive(4, 256, 5e-4, cellular=True)
    csums, ccounts = scene.film()
    cimg = np.zeros(px.shape + (3,))
    cimg[live] = csums[px[live], :3] / ccounts[px[live], None]
    print(json.dumps({"probe": "adaptive", "config": 0, **result, "mean_spp": mean_spp,
                      "rmse_adaptive": rmse_lib.rmse(img, ref, live), "uniform_spp": spp,
                      "rmse_uniform": rmse_lib.rmse(uimg, ref, live), "uniform_ms": c.milliseconds,
                      "cellular": {**cell, "mean_spp": cell["samples"] / (cfg.width * cfg.height), "rmse": rmse_lib.rmse(cimg, ref, live)}}))
    scene.free()
    ctx.close()


def probe_workgrid(args):
    """Config 1 (1920x1080, 64 spp) fed from the work grid by the GPU broker: the progressive order (ranges of 1, 1, 2,
    then 4 samples; GPU-only cells of 64 px, 32 cellular workers) with launches of about one range of the image (32,400
    chunks) and with the whole frame taken at once, beside the uniform wavefront frame; each film audited. Prints the
    frame times and Msamples/s."""
    import x2

    ctx = x2.Context(0)
    s = x2.SyntheticScene(1)
    cfg = s.config
    scene = x2.Scene(ctx, s.desc, cfg)
    pixels = cfg.width * cfg.height
    tiles = ((cfg.width + 7) // 8) * ((cfg.height + 7) // 8)
    out = {"probe": "workgrid", "config": 1, "spp": cfg.spp, "samples": pixels * cfg.spp}
    scene.frame_begin(cfg.spp)
    scene.render_frame_wavefront(0, cfg.spp)  # warm-up
    c = scene.wait()
    scene.frame_begin(cfg.spp)
    scene.render_frame_wavefront(0, cfg.spp)
    c = scene.wait()
    out["uniform_ms"] = c.milliseconds
    for name, want in (("per_range", tiles), ("whole", 1 << 22)):
        grid = x2.WorkGrid(cfg.width, cfg.height, cfg.spp, x2.workgrid_options(samples_per_chunk=4))
        r = scene.render_workgrid(grid, want)
        scene.audit(np.full(pixels, cfg.spp, np.uint32))
        out[name] = {"chunks_per_launch": want, "launches": r["launches"], "ms": r["milliseconds"], "gpu_ms": r["gpu_milliseconds"],
                     "msamples_per_s": r["samples"] / r["milliseconds"] / 1e3}
        grid.free()
    print(json.dumps(out))
    scene.free()
    ctx.close()


def probe(args):
    """One bounded launch for profilers (ncu): `--probe-tiles` evenly spaced tiles of config 1 at 64 spp, in one form;
    the wavefront form without its graph (`--probe-timed`) so each kernel launch is visible on its own."""
    import x2

    if args.probe == "batch":
        return probe_batch(args)
    if args.probe == "volume":
        return probe_volume(args)
    if args.probe == "adjoint":
        return probe_adjoint(args)
    if args.probe == "estimators":
        return probe_estimators(args)
    if args.probe == "forms":
        return probe_forms(args)
    if args.probe == "rmse":
        return probe_rmse(args)
    if args.probe == "adaptive":
        return probe_adaptive(args)
    if args.probe == "workgrid":
        return probe_workgrid(args)
    ctx = x2.Context(0)
    s = x2.SyntheticScene(1)
    cfg = s.config
    scene = x2.Scene(ctx, s.desc, cfg)
    apply_shape(scene, args.shape)
    tiles = ((cfg.width + 7) // 8) * ((cfg.height + 7) // 8)
    sel = np.linspace(0, tiles - 1, args.probe_tiles).astype(np.uint32)
    chunks = np.zeros(len(sel), x2.CHUNK_DTYPE)
    chunks["tile"], chunks["first"], chunks["count"] = sel, 0, cfg.spp
    n = len(sel) * 64 * cfg.spp
    tc = None
    if args.probe == "wavefront" and args.probe_count:
        scene.frame_begin(cfg.spp)
        scene.count_traversal(True)
        scene.launch_wavefront(chunks)
        scene.wait()
        tc = scene.traversal_counts()
        scene.count_traversal(False)
    scene.frame_begin(cfg.spp)
    if args.probe == "plain":
        scene.launch(chunks)
    else:
        scene.wavefront_timing(args.probe_timed)
        scene.launch_wavefront(chunks)
    c = scene.wait()
    out = {"probe": args.probe, "tiles": len(sel), "samples": n, "ms": c.milliseconds, "msamples_per_s": n / c.milliseconds / 1e3,
           "errors": c.errors, "shape": args.shape}
    if args.probe == "wavefront":
        out["kernel_ms"] = scene.wavefront_timing(None)
        out["wavefront"] = scene.wavefront_info()
        if args.probe_timed:
            out["queues"] = scene.wavefront_queues().tolist()  # per iteration: rays extended, shadow rays
        if tc is not None:
            out["traversal"] = tc
            out["simt"] = simt_summary(tc)
    print(json.dumps(out))
    scene.free()
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="x2", choices=["x2", "reference"])
    ap.add_argument("--plain-steps", type=int, default=1)
    ap.add_argument("--skip-plain", action="store_true")
    ap.add_argument("--probe", choices=["plain", "wavefront", "batch", "volume", "adjoint", "rmse", "adaptive", "workgrid", "estimators", "forms"], help="one bounded launch for a profiler, then exit")
    ap.add_argument("--probe-tiles", type=int, default=592)
    ap.add_argument("--probe-timed", action="store_true", help="wavefront probe without its graph (per-kernel launches)")
    ap.add_argument("--probe-count", action="store_true", help="wavefront probe: first an untimed counting launch (node visits, "
                    "triangle tests, traversal lane use)")
    ap.add_argument("--adjoint-only", action="store_true", help="adjoint probe: one primal frame, then one wavefront adjoint launch")
    ap.add_argument("--shape", default="", help="wavefront launch shape fields, e.g. lobe_queues=0,refill=8 (default: the library's)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.probe:
        probe(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run(args)


if __name__ == "__main__":
    main()
