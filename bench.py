"""Benchmark of the per-ray hot path on the 500k-Gaussian scattering showcase workload.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--engine warp|megakernel]

Workload (one "step" = one launch batch of 16 samples per pixel over the whole 512x512 image,
the reference's per-launch granularity, renderer.cpp:32,353-371; 16 steps = the full 256-spp
render): 500k anisotropic Gaussians in value-noise clusters, procedural 2048x1024 HDR
environment with alias-table importance sampling, NEE+MIS with two shadow rays, Russian roulette
from depth 12, max depth 64, isotropic phase.  Metric: Mpaths/s (a path = one (pixel, sample)
camera path run to termination).  Inputs are resident in HBM when the timed region starts; the
L2 is flushed (256 MiB write) between timed steps and each step is timed with CUDA events on the
render stream.  `e2e` times the same metric through the public API from pinned host buffers:
scene + environment upload and build, the whole render, and the image read-back.

Under torchrun each rank renders its own sample range (weak scaling: per-GPU work fixed) and the
per-rank images are reduced over NCCL at the end of the timed region.
`--impl reference` times the reference's path restated on the host cores (oracle port; the
reference itself needs OptiX and an RT-core GPU) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "cuda-volprim_b200"))

METRIC = "Mpaths/s (showcase 500k, NEE+MIS; equal-RMSE vs megakernel = same estimator)"
UNIT = "Mpaths/s"
BATCH_SPP = 16


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=16)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--engine", default="wavefront", choices=["warp", "wavefront", "megakernel"])
    ap.add_argument("--n", type=int, default=500_000)
    ap.add_argument("--res", type=int, default=512)
    ap.add_argument("--spp", type=int, default=256)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-baseline-engine", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the differentiation and serving forms")
    ap.add_argument("--serving-requests", type=int, default=1000)
    ap.add_argument("--rmse-sweep", action="store_true",
                    help="instead of the timed run: RMSE against a high-spp render versus device time, for the "
                         "wavefront and the plain megakernel, and the speed-up at matched RMSE")
    ap.add_argument("--ref-spp", type=int, default=1024, help="samples of the --rmse-sweep reference render")
    return ap.parse_args()


def workload(args):
    from volprim_b200 import scenes
    return scenes.showcase_500k(seed=0, n=args.n, res=args.res, spp=args.spp)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class CpuBaseline:
    """The reference's path restated on the host (oracle port, reference RNG order, CPU BVH) on a
    bounded sample of the workload: pixels drawn from a seeded random permutation of the whole
    image (so every sample covers sky, cloud edge and cloud core in proportion), 2 spp each, all
    host threads.  Successive samples continue the permutation."""

    SPP = 2

    def __init__(self, w):
        import numpy as np
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as O
        self.O, self.w = O, w
        t0 = time.time()
        self.osc = O.OracleScene.from_gaussians(w.gaussians, sigma_multiplier=w.sigma_multiplier, use_bvh=True)
        self.env = O.OracleEnv(w.env) if w.env is not None else O.OracleEnv.constant()
        self.build_s = time.time() - t0
        cfg = w.config
        self.c16 = O.camera16(w.camera, cfg.image_width, cfg.image_height)
        self.threads = O.max_threads()
        self.perm = np.random.default_rng(20240).permutation(cfg.image_width * cfg.image_height)
        self.next = 0

    def sample(self, seconds_target=15.0) -> dict:
        import numpy as np
        cfg = self.w.config
        W = cfg.image_width
        chunk = 4 * self.threads
        spent = trace_s = scan_s = 0.0
        pixels = 0
        while spent < seconds_target and pixels < self.perm.size:
            idx = self.perm[np.arange(self.next, self.next + chunk) % self.perm.size]
            self.next += chunk
            _, secs, tr, sc = self.O.render_pixels(self.osc, self.env, self.c16, cfg, idx % W, idx // W, 0, self.SPP,
                                                   rng_mode="sequential", threads=self.threads)
            spent += secs
            trace_s += tr
            scan_s += sc
            pixels += idx.size
        paths = pixels * self.SPP
        return {"value": paths / spent / 1e6, "unit": UNIT, "cores": self.threads, "kind": "port",
                "scan_fraction": scan_s / max(trace_s, 1e-12),
                "sample": f"{pixels} pixels of a seeded random permutation of the whole {W}x{cfg.image_height} image "
                          f"x {self.SPP} spp, reference RNG order, CPU BVH; {paths} paths in {spent:.1f} s on "
                          f"{self.threads} threads, {100 * scan_s / max(trace_s, 1e-12):.0f}% of the threads' time in "
                          f"the bounce-0 origin-inside scan over all {self.w.gaussians.count} Gaussians "
                          f"(build_origin_inside_set, once per camera path); scene + BVH build "
                          f"{self.build_s:.1f} s untimed"}


def cpu_baseline(w, seconds_target=20.0):
    return CpuBaseline(w).sample(seconds_target)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = workload(args)
    cb = CpuBaseline(w)
    res = []
    for i in range(args.warmup + args.steps):
        r = cb.sample(seconds_target=6.0 if i >= args.warmup else 1.0)
        if i >= args.warmup:
            res.append(r)
    vals = [r["value"] for r in res]
    v = statistics.mean(vals)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators)",
            "config": {"workload": f"showcase_{args.n // 1000}k", "gaussians": args.n, "width": args.res,
                       "height": args.res, "spp_per_rank": args.spp, "nee": "mis", "max_depth": 64, "rr_depth": 12,
                       "env": "procedural 2048x1024", "l2": "n/a (host)"},
            "cpu_baseline": {**res[-1], "value": v},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# Algorithmic bytes of one traversal query's work: a Gaussian's 3-sigma box (2 float4) per box
# test, its whitening record (4 float4) per box hit, a BVH32 inner node (32 child boxes, 64 float4)
# per visit; binary LBVH nodes are 4 float4.
BOX_BYTES, RECORD_BYTES, WIDE_NODE_BYTES, BINARY_NODE_BYTES = 32, 64, 1024, 64
# Per-item path state the wavefront kernels move: extend reads the queue entry, origin, direction,
# key, bounce word and writes albedo + t* (4+16+16+8+4+16); shadow reads the queue entry, origin,
# direction and writes the transmittance (4+16+16+4).
EXTEND_STATE_BYTES, SHADOW_STATE_BYTES = 64, 40


F_CROSS_FLOPS = 111  # FP32 flops of one closed-form chord evaluation (FMA = 2), erf and MUFU excluded
FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12


def l2_copy_gbs(device_bytes=32 << 20, reps=50):
    """Measured L2-resident copy rate: torch copy_ between two 32 MiB buffers (64 MiB, inside the
    126 MB L2), replayed from a captured CUDA graph so launch gaps do not count; read + write bytes
    over CUDA-event time, best of 3."""
    import torch
    a = torch.empty(device_bytes // 4, dtype=torch.float32, device="cuda").fill_(1.0)
    b = torch.empty_like(a)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(3):
            b.copy_(a)
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        for _ in range(reps):
            b.copy_(a)
    best = 0.0
    for _ in range(3):
        g.replay()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        g.replay()
        e1.record()
        e1.synchronize()
        best = max(best, 2 * device_bytes * reps / (e0.elapsed_time(e1) / 1e3) / 1e9)
    del g
    return best


def roofline(args, m, step_stats, sm_mhz=None):
    """Roofline of the dominant kernel, from the counters of one measured batch (m), the CUDA-event
    stage times of the timed steps (the steps are the same batch size over the same image) and the
    per-unit ncu figures of profiles/traffic.json (warp instructions and DRAM bytes per unit).

    The traversal kernels are issue-bound (the scene is L2-resident, DRAM runs below 1% of peak),
    so the binding roof is the SMs' issue rate: 148 SMs x 4 schedulers x one warp instruction per
    cycle at the SM clock sampled during the timed region.  The bytes the traversal touches are
    reported against a measured L2 copy rate (l2_demand) and the DRAM bytes against the measured
    HBM copy rate (hbm)."""
    peak_hbm, peak_kind = measured_peaks()

    def query_bytes(k):
        node = BINARY_NODE_BYTES if args.engine == "megakernel" else WIDE_NODE_BYTES
        return m["query_prim_tests"][k] * BOX_BYTES + m["query_geo_loads"][k] * RECORD_BYTES + m["query_nodes"][k] * node

    n = len(step_stats)
    if args.engine == "wavefront":
        ms = [sum(st["ms_stage"][k] for st in step_stats) / n for k in range(3)]
        nl = [sum(st["stage_launches"][k] for st in step_stats) / n for k in range(3)]
        kern = [("k_wf_extend", query_bytes(0) + query_bytes(2) + m["bounces"] * EXTEND_STATE_BYTES,
                 "free-flight argmin + scatter-point albedo", m["bounces"], "path bounces", EXTEND_STATE_BYTES),
                ("k_wf_shadow", query_bytes(1) + m["shadow_rays"] * SHADOW_STATE_BYTES,
                 "transmittance (NEE shadow rays)", m["shadow_rays"], "shadow rays", SHADOW_STATE_BYTES)]
        k = 0 if ms[0] >= ms[1] else 1
        name, alg, what, units, unit_name, state_bytes = kern[k]
        step_ms, launches = ms[k], nl[k]
        share = ms[k] / max(1e-9, sum(st["ms_kernels"] for st in step_stats) / n)
    else:
        name = "k_render_mega" if args.engine == "megakernel" else "k_render_warp"
        alg = query_bytes(0) + query_bytes(1) + query_bytes(2)
        what, units, unit_name, state_bytes = "whole path loop", m["paths"], "paths", None
        step_ms = sum(st["ms_kernels"] for st in step_stats) / n
        launches, share = 1, 1.0
    sec_per_launch = step_ms / launches / 1e3
    units_per_launch = units / launches
    prof = {}
    traffic_file = ROOT / "profiles" / "traffic.json"
    if traffic_file.exists():
        try:
            prof = json.loads(traffic_file.read_text()).get(name) or {}
        except (ValueError, TypeError):
            prof = {}
    clock = sm_mhz or 1965.0
    issue_peak = 148 * 4 * clock * 1e6 / 1e9  # G warp-instructions / s
    inst = prof.get("warp_inst_per_unit")
    traffic = prof["dram_bytes_per_unit"] * units_per_launch if prof.get("dram_bytes_per_unit") else None
    l2_peak = l2_copy_gbs()
    l2_achieved = alg / launches / sec_per_launch / 1e9
    roof = {"kernel": name, "kernel_work": what, "kernel_share_of_step": share, "launches_per_step": launches,
            "kernel_ms_per_launch": step_ms / launches, "units_per_launch": units_per_launch, "units": unit_name}
    if inst:
        achieved = inst * units_per_launch / sec_per_launch / 1e9
        roof.update({"bound": "issue", "achieved": achieved, "peak": issue_peak, "unit": "G warp-instructions/s",
                     "frac": achieved / issue_peak,
                     "peak_source": f"148 SMs x 4 schedulers x 1 warp-instruction/cycle x {clock:.0f} MHz "
                                    f"({'median SM clock sampled in the timed region' if sm_mhz else 'max clock'})",
                     "warp_instructions_per_unit": inst, "instructions_source": prof.get("source")})
    else:
        roof.update({"bound": "issue", "achieved": None, "peak": issue_peak, "unit": "G warp-instructions/s",
                     "frac": None, "note": "no ncu instruction count per unit in profiles/traffic.json"})
    roof["traffic"] = traffic
    roof["traffic_source"] = prof.get("source")
    roof["traffic_per_unit"] = prof.get("dram_bytes_per_unit")
    roof["declared_state_bytes_per_unit"] = state_bytes
    roof["l2_demand"] = {"achieved": l2_achieved, "peak": l2_peak, "unit": "GB/s", "frac": l2_achieved / l2_peak,
                         "algorithmic_bytes_per_launch": alg / launches,
                         "peak_source": "measured: L2-resident torch copy, 2 x 32 MiB, read + write bytes",
                         "note": "3-sigma boxes tested x 32 B + Gaussian records loaded x 64 B + BVH32 inner nodes "
                                 "x 1 KiB + per-item path state, per launch, over its CUDA-event time; the 70 MB "
                                 "scene is L2-resident and L1 serves about half of the requests (ncu L1 hit rate "
                                 "54-60%), so frac can exceed 1"}
    if traffic is not None:
        roof["hbm"] = {"achieved": traffic / sec_per_launch / 1e9, "peak": peak_hbm, "unit": "GB/s",
                       "frac": traffic / sec_per_launch / 1e9 / peak_hbm, "peak_source": peak_kind}
    roof["per_step"] = {"crossings": m["crossings"], "bounces": m["bounces"], "shadow_rays": m["shadow_rays"],
                        "query_nodes[argmin,tau,albedo]": m["query_nodes"],
                        "query_leaves[argmin,tau,albedo]": m["query_leaves"],
                        "query_box_tests[argmin,tau,albedo]": m["query_prim_tests"],
                        "query_record_loads[argmin,tau,albedo]": m["query_geo_loads"],
                        "max_point_overlap": m["max_point_overlap"], "max_hits_per_ray": m["max_hits_per_ray"]}
    if args.engine == "wavefront":
        roof["stage_ms_per_step[extend,shadow,other]"] = ms
    # The FP32 side: closed-form (ray, Gaussian) evaluations of the step's traversal kernels times
    # the declared 111 FP32 flops each (FMA = 2; erf and MUFU work not counted), against the
    # nominal FP32 rate (148 SMs x 128 lanes x 2 flops x 1965 MHz) -- no FP32 peak is measured.
    trav_ms = (ms[0] + ms[1]) if args.engine == "wavefront" else step_ms
    fp32_tflops = m["crossings"] * F_CROSS_FLOPS / (trav_ms / 1e3) / 1e12
    roof["fp32_side"] = {"crossings_per_step": m["crossings"], "flops_per_crossing": F_CROSS_FLOPS,
                         "achieved_tflops": fp32_tflops, "nominal_peak_tflops": FP32_NOMINAL_TFLOPS,
                         "frac": fp32_tflops / FP32_NOMINAL_TFLOPS, "peak_source": "nominal"}
    return roof


def run_ours(args):
    import numpy as np
    import torch
    import volprim_b200 as vp
    from volprim_b200 import _capi

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))

    w = workload(args)
    cfg = w.config
    cfg.engine = args.engine
    cfg.batch_spp = BATCH_SPP
    # weak scaling: every rank renders its own `spp` samples of a world*spp-sample image
    cfg.num_samples_per_pixel = args.spp * world
    W, H = cfg.image_width, cfg.image_height
    ctx = vp.Context(local)
    scene = vp.Scene(ctx, w.gaussians, w.sigma_multiplier)
    env = vp.Environment(ctx, rgb=w.env)
    img = vp.ProgressiveImage(ctx, W, H)
    stream = torch.cuda.ExternalStream(ctx.stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    from volprim_b200 import distributed as D
    base, _ = D.sample_range(rank, world, args.spp)

    tcfg = vp.Config(**{**cfg.__dict__, "time_stages": True})  # CUDA events around the traversal kernels

    def step(i):  # one launch batch of BATCH_SPP samples
        off = base + (i * BATCH_SPP) % args.spp
        return img.accumulate(scene, env, w.camera, tcfg, off, BATCH_SPP)

    def new_render_starts(i):  # steps past spp/BATCH_SPP begin a fresh render of the same image
        return i > 0 and (i * BATCH_SPP) % args.spp == 0

    # warm-up (also the first steps of the image)
    for i in range(args.warmup):
        step(i)
    # measured counters of one batch (untimed): crossings, node visits, Gaussian tests
    mcfg = vp.Config(**{**cfg.__dict__, "measure_caps": True})
    img_m = vp.ProgressiveImage(ctx, W, H)
    mstats = img_m.accumulate(scene, env, w.camera, mcfg, base, BATCH_SPP)
    img_m.close()
    img.clear()

    clocks = ClockSampler(local)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    t_wall = time.perf_counter()
    step_stats = []
    for i in range(args.steps):
        if new_render_starts(i):
            img.clear()  # outside the step's events: each spp/16 consecutive steps are one full render
        with torch.cuda.stream(stream):
            flush.fill_(float(i))  # L2 flush, outside the step's events
            starts[i].record(stream)
        step_stats.append(step(i))
        with torch.cuda.stream(stream):
            ends[i].record(stream)
    reduce_ms = 0.0
    if dist:  # the job's one exchange: count-weighted mean of the per-rank images
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        acc = torch.empty((H, W, 4), dtype=torch.float32, device="cuda")
        ev0.record(stream)
        _capi.check(_capi.lib.vp_image_read(img.handle, acc.data_ptr(), _capi.VP_MEMORY_DEVICE))
        with torch.cuda.stream(stream):
            acc = D.combine(acc, BATCH_SPP * args.steps)
            ev1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t_wall
    clk = clocks.stop()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    if dist:
        reduce_ms = ev0.elapsed_time(ev1)
    total_ms = sum(step_ms) + reduce_ms
    if dist:
        t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    paths_per_rank = W * H * BATCH_SPP * args.steps
    value = paths_per_rank * world / (total_ms / 1e3) / 1e6
    ms_per_step = total_ms / args.steps

    roof = roofline(args, mstats, step_stats, clk.get("sm_mhz"))
    launches = sum(st["launches"] for st in step_stats)

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generators)",
            "config": {"workload": f"showcase_{args.n // 1000}k", "gaussians": args.n, "width": W, "height": H,
                       "spp_per_rank": args.spp,
                       "step": f"{BATCH_SPP} spp over the full image; every {args.spp // BATCH_SPP} consecutive steps "
                               f"are one complete {args.spp}-spp render (the image is cleared, untimed, between renders)",
                       "nee": "mis",
                       "max_depth": cfg.max_bounces, "rr_depth": cfg.rr_depth, "env": "procedural 2048x1024",
                       "engine": args.engine, "precision": "fast (FP32)",
                       "l2": "flushed (256 MiB write) between timed steps", "parallelism": f"samples x{world}"},
            "clocks": clk, "gpu_launches": launches, "roofline": roof,
            "scene": scene.info(), "env_build_ms": env.build_ms, "wall_s": wall}
    if rank == 0 and not args.no_baseline_engine and args.engine != "megakernel" and world == 1:
        # The plain per-pixel megakernel of the same method on the same batches (for the ratio):
        # over the Karras LBVH binary tree (the straightforward build), and over the same PLOC
        # tree as the wavefront (the ratio with tree quality held equal).
        mcfg2 = vp.Config(**{**cfg.__dict__, "engine": "megakernel"})

        def mega_ms(sc):
            im2 = vp.ProgressiveImage(ctx, W, H)
            im2.accumulate(sc, env, w.camera, mcfg2, 0, BATCH_SPP)
            torch.cuda.synchronize()
            ms = []
            for i in range(2):
                st = im2.accumulate(sc, env, w.camera, mcfg2, BATCH_SPP * (i + 1), BATCH_SPP)
                ms.append(st["ms_kernels"])
            im2.close()
            return statistics.mean(ms)

        lbvh_scene = vp.Scene(ctx, w.gaussians, w.sigma_multiplier, binary_builder="lbvh")
        ms_l = mega_ms(lbvh_scene)
        lbvh_scene.close()
        ms_p = mega_ms(scene)
        line["megakernel_baseline"] = {"value": W * H * BATCH_SPP / (ms_l / 1e3) / 1e6, "unit": UNIT,
                                       "ms_per_step": ms_l, "tree": "Karras LBVH (binary radix tree over Morton codes)"}
        line["megakernel_same_tree"] = {"value": W * H * BATCH_SPP / (ms_p / 1e3) / 1e6, "unit": UNIT,
                                        "ms_per_step": ms_p, "tree": "PLOC clustering (the wavefront's binary tree)"}
    if not args.no_e2e and world == 1:
        line["e2e"] = e2e_run(args, w, local)
    if rank == 0 and not args.no_forms and world == 1:
        line["differentiation"] = differentiation_form(local)
        line["serving"] = serving_form(local, args.serving_requests)
        line["other_configs"] = other_configs(local)
    if rank == 0 and not args.no_cpu and world == 1:
        line["cpu_baseline"] = cpu_baseline(w)
    if rank == 0:
        print(json.dumps(line), flush=True)
    img.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def e2e_run(args, w, device):
    """Public API end to end from pinned host memory: scene + env upload and device builds, the full
    render, read-back of the image; Mpaths/s over the whole job."""
    import numpy as np
    import torch
    import volprim_b200 as vp

    def pinned(a):
        t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).pin_memory()
        return t.numpy()

    g = w.gaussians
    gp = vp.Gaussians(pinned(g.mean), pinned(g.scale), pinned(g.quat_wxyz), pinned(g.density), pinned(g.albedo))
    envp = pinned(w.env)
    cfg = vp.Config(**{**w.config.__dict__, "num_samples_per_pixel": args.spp, "batch_spp": BATCH_SPP,
                       "engine": args.engine})
    ctx = vp.Context(device)
    times = []
    for rep in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = vp.Renderer(cfg, gp, w.camera, env=envp, sigma_multiplier=w.sigma_multiplier, ctx=ctx)
        out = r.render()
        times.append(time.perf_counter() - t0)
        r.scene.close()
        r.env.close()
    paths = cfg.image_width * cfg.image_height * cfg.num_samples_per_pixel
    h2d = sum(a.nbytes for a in (gp.mean, gp.scale, gp.quat_wxyz, gp.density, gp.albedo)) + envp.nbytes
    return {"value": paths / min(times) / 1e6, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(out.nbytes), "seconds": min(times),
            "note": "one step here = the whole job (upload, BVH + env builds, 256 spp, read-back)"}


def differentiation_form(device):
    """grad/s of the differentiation workload (100k Gaussians, absorption + emission, 4 cameras at
    256x256 x 8 spp, L2 loss against a render of perturbed parameters): one gradient = the
    autograd Function's scene build + 4 forward renders + 4 adjoint renders, timed on the host
    around torch.cuda.synchronize (the library calls are synchronous)."""
    import numpy as np
    import torch
    import volprim_b200 as vp
    from volprim_b200 import _capi, scenes
    from volprim_b200.autograd import EmissionRender, render_emission_images
    from volprim_b200.emission import render_emission

    w = scenes.emission_100k()
    ctx = vp.Context(device)
    env = vp.Environment(ctx, constant=w.env_constant)
    dev = torch.device("cuda", device)
    tg, te = scenes.perturbed(w)
    ts = vp.Scene(ctx, tg, w.sigma_multiplier)
    ts.set_emission(te)
    target = torch.stack([torch.from_numpy(render_emission(ts, env, c, w.config)[..., :3]) for c in w.cameras]).to(dev)
    ts.close()
    g = w.gaussians
    t = [torch.tensor(np.asarray(a, np.float32), device=dev, requires_grad=True)
         for a in (g.mean, g.scale, g.quat_wxyz, g.density, w.emission)]

    def one():
        for x in t:
            x.grad = None
        imgs = render_emission_images(*t, w.cameras, w.config, env, w.sigma_multiplier, ctx)
        loss = ((imgs - target) ** 2).sum()
        loss.backward()
        torch.cuda.synchronize()
        return float(loss)

    one()
    one()
    times, splits = [], []
    for _ in range(7):
        t0 = time.perf_counter()
        one()
        times.append(time.perf_counter() - t0)
        splits.append(dict(EmissionRender.last_ms))
    env.close()
    ctx.close()
    paths = len(w.cameras) * w.config.image_width * w.config.image_height * w.config.num_samples_per_pixel
    med = statistics.median(times)
    split = {k: statistics.median(s[k] for s in splits) for k in splits[0]}
    return {"metric": "grad/s", "value": 1.0 / med, "unit": "grad/s",
            "ms_per_grad": 1e3 * med, "ms_per_grad_min": 1e3 * min(times), "timed_gradients": len(times),
            "workload": "emission_100k (100k Gaussians, 4 cameras, "
            "256x256, 8 spp, FAST)", "paths_per_forward": paths,
            "scene_build_ms": split["scene_build"], "forward_kernel_ms": split["forward_kernels"],
            "backward_kernel_ms": split["backward_kernels"],
            "note": "one gradient = scene build from the parameter tensors + 4 forward + 4 adjoint renders "
                    "(autograd Function), host-timed around torch.cuda.synchronize: median of 7 after 2 warm-up "
                    "gradients (the host loop is sensitive to other load on the host); scene build, forward and "
                    "adjoint kernel times are CUDA-event times inside the same timed gradients (medians)"}


def other_configs(device):
    """The other two configurations (wavefront engine, inputs resident):
    * the 256-Gaussian absorption case (128x128, 16 spp), in AUTO precision (the ACCURATE
      float-pair set-up this albedo-0 scene selects) and in FAST, both FP32 arithmetic: 5 timed
      renders each (median, min, max);
    * the 2M-Gaussian traversal stress case at its stated size (1024x1024, all 64 spp as four
      16-spp batches, timed twice), its BVH build time (3 builds) and, from one measured 16-spp
      batch, the per-query chord-count histograms (power-of-two bins) behind its overlap and
      hit maxima."""
    import torch
    import volprim_b200 as vp
    from volprim_b200 import scenes

    def spread(v):
        return {"median": statistics.median(v), "min": min(v), "max": max(v), "runs": len(v)}

    out = {}
    ctx = vp.Context(device)
    w = scenes.absorption_256()
    cfg = w.config
    cfg.engine = "wavefront"
    sc = vp.Scene(ctx, w.gaussians, w.sigma_multiplier)
    env = vp.Environment(ctx, constant=(1.0, 1.0, 1.0))
    img = vp.ProgressiveImage(ctx, cfg.image_width, cfg.image_height)
    for prec in ("auto", "fast"):
        c = vp.Config(**{**cfg.__dict__, "precision": prec})
        img.accumulate(sc, env, w.camera, c, 0, cfg.num_samples_per_pixel)  # warm-up
        rates, ms = [], []
        for _ in range(5):
            img.clear()
            torch.cuda.synchronize()
            st = img.accumulate(sc, env, w.camera, c, 0, cfg.num_samples_per_pixel)
            rates.append(st["paths"] / (st["ms_kernels"] / 1e3) / 1e6)
            ms.append(st["ms_kernels"])
        out["absorption_256" if prec == "auto" else "absorption_256_fast"] = {
            "mpaths_per_s": statistics.median(rates), "mpaths_per_s_spread": spread(rates), "ms": statistics.median(ms),
            "paths": st["paths"], "gaussians": sc.info()["count"],
            "precision": "auto = ACCURATE: FP32 with float-pair set-up and sums" if prec == "auto" else
                         "FAST: FP32, hardware exp/log approximations"}
    img.close()
    env.close()
    sc.close()

    w = scenes.stress_2m()
    cfg = w.config
    cfg.engine = "wavefront"
    builds = []
    for _ in range(3):
        sc = vp.Scene(ctx, w.gaussians, w.sigma_multiplier)
        builds.append(sc.info()["build_ms"])
        if len(builds) < 3:
            sc.close()
    env = vp.Environment(ctx, rgb=w.env)
    img = vp.ProgressiveImage(ctx, cfg.image_width, cfg.image_height)
    spp = cfg.num_samples_per_pixel
    img.accumulate(sc, env, w.camera, cfg, 0, BATCH_SPP)  # warm-up
    rates, totals = [], []
    for _ in range(2):
        img.clear()
        torch.cuda.synchronize()
        ms = paths = 0
        for off in range(0, spp, BATCH_SPP):
            st = img.accumulate(sc, env, w.camera, cfg, off, BATCH_SPP)
            ms += st["ms_kernels"]
            paths += st["paths"]
        rates.append(paths / (ms / 1e3) / 1e6)
        totals.append(ms)
    mcfg = vp.Config(**{**cfg.__dict__, "measure_caps": True})
    img.clear()
    m = img.accumulate(sc, env, w.camera, mcfg, 0, BATCH_SPP)
    info = sc.info()
    out["stress_2m"] = {"mpaths_per_s": statistics.median(rates), "mpaths_per_s_spread": spread(rates),
                        "ms_per_render": statistics.median(totals), "spp": spp, "paths": paths,
                        "gaussians": info["count"], "bvh_build_ms": statistics.median(builds),
                        "bvh_build_ms_spread": spread(builds), "bvh32_nodes": info["wide_nodes"], "tau_order": info["tau_order"],
                        "precision": cfg.precision,
                        "max_point_overlap": m["max_point_overlap"], "max_hits_per_ray": m["max_hits_per_ray"],
                        "crossings_per_16spp": m["crossings"],
                        "chords_per_query_hist": {
                            "bins": "0, [1,2), [2,4), ..., [2^13, 2^14), >= 2^14",
                            "argmin": m["hits_hist"][0], "transmittance": m["hits_hist"][1],
                            "sample": "one measured 16-spp batch of the 1024x1024 image"}}
    img.close()
    env.close()
    sc.close()
    ctx.close()
    return out


SERVING_P99_TARGET_S = 3.0  # the stated p99 latency target of the serving form, at 80% of offline throughput


def serving_form(device, n_requests):
    """The serving workload (volprim_b200.serving.serving_study) on its 4 resident scenes
    (50k / 100k / 250k / 500k Gaussians, seeds 1-4): offline capacity (one vp_render per request,
    back to back) and served capacity on the first 300 requests of the seeded stream at t = 0;
    then `n_requests` with Poisson arrivals at 80% of the offline capacity, served (SRPT) and
    through the plain per-request loop on the same arrivals (p50 / p99 latency)."""
    import volprim_b200 as vp
    from volprim_b200.serving import serving_study

    ctx = vp.Context(device)
    res = serving_study(ctx, n_requests=n_requests, capacity_requests=min(300, n_requests), load=0.8,
                        schedules=("srpt",))
    ctx.close()
    served, plain, cap = res["served"]["srpt"], res["plain"], res["served_capacity"]["srpt"]
    return {"metric": "p50/p99 request latency", "unit": "s", "p50_s": served["p50_s"], "p90_s": served["p90_s"],
            "p99_s": served["p99_s"], "max_s": served["max_s"], "p99_target_s": SERVING_P99_TARGET_S,
            "meets_p99_target": served["p99_s"] <= SERVING_P99_TARGET_S,
            "mpaths_per_s": served["mpaths_per_s"],
            "offline_mpaths_per_s": res["offline_mpaths_per_s"],
            "served_capacity_mpaths_per_s": cap["mpaths_per_s"],
            "capacity_fraction_of_offline": cap["fraction_of_offline"],
            "served_device_busy_at_capacity": cap["device_busy"],
            "arrival_rate_per_s": res["arrival_rate_per_s"], "load_of_offline": res["load"],
            "requests": n_requests, "capacity_requests": res["capacity_requests"],
            "mean_paths_per_request": res["mean_paths_per_request"],
            "plain_per_request": {k: plain[k] for k in ("p50_s", "p90_s", "p99_s", "max_s", "mpaths_per_s")},
            "workload": "4 resident scenes (50k/100k/250k/500k Gaussians), requests: resolution in "
                        "{64,128,256,512}^2, spp in {1,4,16,64}, random camera at distance 3.5; Poisson arrivals at "
                        "80% of the offline capacity (plain per-request loop at t = 0); 150 GB budget; SRPT "
                        "schedule (half the free slots kept for the oldest request), 2^18 path slots"}


def rmse_sweep(args):
    """Equal-RMSE comparison by measurement: each engine renders the showcase progressively in
    16-spp batches; after each batch its RMSE against an independent high-spp render (other seed,
    wavefront) and its cumulative device time are recorded.  At every RMSE level the wavefront
    reaches, the megakernel's time is interpolated on log(time) vs log(RMSE); the speed-up at
    matched RMSE is their ratio.  The reference's own noise adds the same variance to both curves."""
    import numpy as np
    import volprim_b200 as vp

    w = workload(args)
    cfg = w.config
    cfg.batch_spp = BATCH_SPP
    W, H = cfg.image_width, cfg.image_height
    ctx = vp.Context(0)
    scene = vp.Scene(ctx, w.gaussians, w.sigma_multiplier)
    env = vp.Environment(ctx, rgb=w.env)
    ref_cfg = vp.Config(**{**cfg.__dict__, "seed": cfg.seed + 1000, "num_samples_per_pixel": args.ref_spp,
                           "engine": "wavefront"})
    ref_img = vp.ProgressiveImage(ctx, W, H)
    for off in range(0, args.ref_spp, 64):
        ref_img.accumulate(scene, env, w.camera, ref_cfg, off, min(64, args.ref_spp - off))
    ref = ref_img.read()[..., :3].astype(np.float64)
    ref_img.close()

    def curve(engine, sc):
        c = vp.Config(**{**cfg.__dict__, "engine": engine})
        im = vp.ProgressiveImage(ctx, W, H)
        im.accumulate(sc, env, w.camera, c, 0, BATCH_SPP)  # warm-up batch, then start again
        im.clear()
        pts, t = [], 0.0
        for off in range(0, args.spp, BATCH_SPP):
            t += im.accumulate(sc, env, w.camera, c, off, BATCH_SPP)["ms_kernels"]
            rmse = float(np.sqrt(np.mean((im.read()[..., :3] - ref) ** 2)))
            pts.append({"spp": off + BATCH_SPP, "ms": t, "rmse": rmse})
        im.close()
        return pts

    wave = curve("wavefront", scene)
    lbvh = vp.Scene(ctx, w.gaussians, w.sigma_multiplier, binary_builder="lbvh")
    mega = curve("megakernel", lbvh)
    lbvh.close()
    lr_m = np.log([p["rmse"] for p in mega])
    lt_m = np.log([p["ms"] for p in mega])
    order = np.argsort(lr_m)
    matched = []
    for p in wave:
        lr = math.log(p["rmse"])
        if lr_m.min() <= lr <= lr_m.max():
            t_m = float(np.exp(np.interp(lr, lr_m[order], lt_m[order])))
            matched.append({"rmse": p["rmse"], "wavefront_ms": p["ms"], "megakernel_ms": t_m,
                            "speedup": t_m / p["ms"]})
    scale = float(np.sqrt(np.mean(ref ** 2)))
    ratio = [m["rmse"] / p["rmse"] for p, m in zip(wave, mega)]  # same estimator and random numbers
    line = {"metric": "speed-up at matched RMSE (wavefront vs plain per-pixel megakernel over the Karras LBVH)",
            "value": statistics.median([m["speedup"] for m in matched]) if matched else None, "unit": "x",
            "higher_is_better": True,
            "config": {"workload": f"showcase_{args.n // 1000}k", "width": W, "height": H, "spp": args.spp,
                       "reference": f"wavefront, {args.ref_spp} spp, seed {ref_cfg.seed}", "rms_of_reference": scale},
            "rmse_ratio_megakernel_over_wavefront_at_equal_spp": {"min": min(ratio), "max": max(ratio)},
            "time_ratio_at_equal_spp": mega[-1]["ms"] / wave[-1]["ms"],
            "wavefront": wave, "megakernel": mega, "matched": matched}
    print(json.dumps(line), flush=True)
    scene.close()


def main():
    args = parse()
    if args.rmse_sweep:
        rmse_sweep(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
