"""Serving over the C ABI (vp_server_*): several scenes resident on the device, a request FIFO
admitted by a device-memory budget, and continuous batching of every admitted request's paths
into the same wavefront launches (replayed as a captured CUDA graph).

`make_trace` builds the serving workload's request stream (Poisson arrivals; scene, square
resolution and spp drawn uniformly; a random camera on a sphere around the scene) and
`run_trace` replays it in real time against a Server, recording each request's latency from its
arrival to the moment the host sees it complete.  `run_trace_plain` replays the same stream with
one vp_render call per request in arrival order (the plain per-request launch).
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass

import numpy as np

from . import _capi
from ._capi import check, lib
from .api import Camera, Config, Context, Environment, Scene, _alive, _is_cuda_tensor, _sync_torch


class Server:
    """vp_server_create / add_scene / submit / step / poll."""

    def __init__(self, ctx: Context, memory_budget_bytes: int = 150 * 10 ** 9, path_slots: int = 1 << 18,
                 max_requests: int = 256, iterations_per_step: int = 4, precision: str = "fast",
                 use_graph: bool = True, schedule: str = "fifo", srpt_reserve: float = 0.5, lanes: int = 1,
                 srpt_aging: float = 0.0):
        c = _capi.vp_server_config()
        c.memory_budget_bytes = int(memory_budget_bytes)
        c.path_slots = int(path_slots)
        c.max_requests = int(max_requests)
        c.iterations_per_step = int(iterations_per_step)
        c.precision = {"auto": 0, "fast": 1, "accurate": 2}[precision]
        c.use_graph = 1 if use_graph else 0
        c.schedule = {"fifo": 0, "fair": 1, "srpt": 2}[schedule]
        c.srpt_reserve = float(srpt_reserve)
        c.lanes = int(lanes)
        c.srpt_aging = float(srpt_aging)
        h = C.c_void_p()
        check(lib.vp_server_create(ctx.handle, C.byref(c), C.byref(h)))
        self.handle, self.ctx = h, ctx
        self._outs = {}

    def add_scene(self, scene: Scene, env: Environment) -> int:
        sid = C.c_uint32()
        check(lib.vp_server_add_scene(self.handle, scene.handle, env.handle, C.byref(sid)))
        return sid.value

    def submit(self, scene_id: int, camera: Camera, config: Config, out=None) -> int:
        """Queues a request; its (H, W, 4) mean image lands in `out` (a host array or a CUDA
        tensor; a new host array when None) when it completes.  Returns the request id."""
        r = _capi.vp_request()
        r.scene_id = int(scene_id)
        r.camera = camera.to_c()
        r.params = config.to_c()
        shape = (config.image_height, config.image_width, 4)
        if out is None:
            out = np.empty(shape, np.float32)
        if _is_cuda_tensor(out):
            if not out.is_contiguous() or tuple(out.shape) != shape:
                raise ValueError("out must be a contiguous (H, W, 4) float32 CUDA tensor")
            _sync_torch(out)
            r.out_rgba, r.memory = out.data_ptr(), _capi.VP_MEMORY_DEVICE
        else:
            if out.dtype != np.float32 or not out.flags.c_contiguous or out.shape != shape:
                raise ValueError("out must be a contiguous (H, W, 4) float32 array")
            r.out_rgba, r.memory = out.ctypes.data, _capi.VP_MEMORY_HOST
        rid = C.c_uint64()
        check(lib.vp_server_submit(self.handle, C.byref(r), C.byref(rid)))
        self._outs[rid.value] = out
        return rid.value

    def step(self) -> int:
        n = C.c_uint32()
        check(lib.vp_server_step(self.handle, C.byref(n)))
        return n.value

    def cancel(self, request_id: int) -> None:
        """vp_server_cancel: the request is never delivered and its output is never written."""
        check(lib.vp_server_cancel(self.handle, C.c_uint64(request_id)))
        self._outs.pop(request_id, None)

    def inject_alloc_failures(self, n: int) -> None:
        """vp_server_inject_alloc_failures: the next n accumulator allocations fail (host-side
        fault injection for tests)."""
        check(lib.vp_server_inject_alloc_failures(self.handle, C.c_uint32(n)))

    def poll(self) -> list:
        ids = (C.c_uint64 * 1024)()
        out = []
        while True:
            n = C.c_uint32()
            check(lib.vp_server_poll(self.handle, ids, 1024, C.byref(n)))
            out.extend(ids[i] for i in range(n.value))
            if n.value < 1024:
                return out

    def result(self, request_id: int):
        """The output buffer of a completed request (released from the server's bookkeeping)."""
        return self._outs.pop(request_id)

    def stats(self) -> dict:
        s = _capi.vp_server_stats()
        check(lib.vp_server_get_stats(self.handle, C.byref(s)))
        return {k: getattr(s, k) for k, _ in s._fields_}

    def close(self):
        if getattr(self, "handle", None):
            if _alive(self.ctx):
                lib.vp_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class Request:
    arrival: float          # seconds from the trace start
    scene_id: int
    camera: Camera
    config: Config

    @property
    def paths(self) -> int:
        c = self.config
        return c.image_width * c.image_height * c.num_samples_per_pixel


def random_camera(rng: np.random.Generator, distance: float = 3.5, vfov: float = 40.0) -> Camera:
    v = rng.normal(size=3)
    v /= np.linalg.norm(v)
    up = (0.0, 1.0, 0.0) if abs(v[1]) < 0.95 else (0.0, 0.0, 1.0)
    return Camera.perspective(tuple(float(x) for x in distance * v), (0.0, 0.0, 0.0), up, vfov)


def make_trace(seed: int, n: int, rate: float, n_scenes: int, resolutions=(64, 128, 256, 512),
               spps=(1, 4, 16, 64), max_bounces: int = 64) -> list:
    """n requests with exponential inter-arrival times of mean 1/rate: scene, square resolution and
    spp uniform over the given choices, camera uniform on the sphere of radius 3.5 looking at the
    origin, the scattering controls of the 500k showcase (MIS NEE, isotropic phase, roulette from
    depth 12), seed = request index."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += float(rng.exponential(1.0 / rate)) if rate > 0 else 0.0
        res = int(rng.choice(resolutions))
        spp = int(rng.choice(spps))
        cfg = Config(num_samples_per_pixel=spp, image_width=res, image_height=res, seed=i, hg_g=0.0,
                     max_bounces=max_bounces, rr_depth=12, nee="mis", precision="fast", batch_spp=16)
        out.append(Request(t, int(rng.integers(n_scenes)), random_camera(rng), cfg))
    return out


def percentile(values, q: float) -> float:
    """The q-th percentile (nearest rank on the sorted values)."""
    v = sorted(values)
    if not v:
        return float("nan")
    k = max(0, min(len(v) - 1, int(math.ceil(q / 100.0 * len(v))) - 1))
    return float(v[k])


def run_trace(server: Server, trace: list, keep_outputs: bool = False, out_factory=None) -> dict:
    """Replays the trace in real time: each request is submitted once its arrival time has passed,
    the server steps while anything is pending or active, and a request's latency runs from its
    arrival to the step that completes it.  Returns latencies (s), makespan, paths and (optional)
    outputs by trace index."""
    t0 = time.perf_counter()
    nxt = 0
    ids = {}
    lat = [None] * len(trace)
    outs = {}
    remaining = len(trace)
    while remaining:
        now = time.perf_counter() - t0
        while nxt < len(trace) and trace[nxt].arrival <= now:
            r = trace[nxt]
            out = out_factory(r) if out_factory else None
            ids[server.submit(r.scene_id, r.camera, r.config, out)] = nxt
            nxt += 1
        st = server.stats()
        if st["active"] == 0 and st["pending"] == 0:
            if nxt < len(trace):  # idle until the next arrival
                time.sleep(max(0.0, trace[nxt].arrival - (time.perf_counter() - t0)))
            continue
        server.step()
        done_t = time.perf_counter() - t0
        for rid in server.poll():
            k = ids.pop(rid)
            lat[k] = done_t - trace[k].arrival
            o = server.result(rid)
            if keep_outputs:
                outs[k] = o
            remaining -= 1
    makespan = time.perf_counter() - t0
    paths = sum(r.paths for r in trace)
    return {"latency_s": lat, "makespan_s": makespan, "paths": paths, "outputs": outs,
            "p50_s": percentile(lat, 50), "p99_s": percentile(lat, 99),
            "mpaths_per_s": paths / makespan / 1e6, "server": server.stats()}


def run_trace_plain(scenes: list, envs: list, trace: list) -> dict:
    """The same stream through one vp_render per request, in arrival order (a request starts when
    it has arrived and the previous one has finished)."""
    t0 = time.perf_counter()
    lat = []
    busy = 0.0
    for r in trace:
        now = time.perf_counter() - t0
        if r.arrival > now:
            time.sleep(r.arrival - now)
        a = time.perf_counter()
        p = r.config.to_c()
        cam = r.camera.to_c()
        out = np.empty((r.config.image_height, r.config.image_width, 4), np.float32)
        st = _capi.vp_render_stats()
        check(lib.vp_render(scenes[r.scene_id].handle, envs[r.scene_id].handle, C.byref(cam), C.byref(p),
                            out.ctypes.data, _capi.VP_MEMORY_HOST, C.byref(st)))
        b = time.perf_counter()
        busy += b - a
        lat.append(b - t0 - r.arrival)
    makespan = time.perf_counter() - t0
    paths = sum(r.paths for r in trace)
    return {"latency_s": lat, "makespan_s": makespan, "paths": paths, "busy_s": busy,
            "p50_s": percentile(lat, 50), "p99_s": percentile(lat, 99), "mpaths_per_s": paths / makespan / 1e6}


def capacity(trace: list) -> list:
    """The trace with every arrival at t = 0 (saturation)."""
    return [Request(0.0, r.scene_id, r.camera, r.config) for r in trace]


def schedule_spec(spec: str) -> tuple:
    """A schedule name of the serving study: "fifo", "fair", "srpt", or "srpt/A" for SRPT with
    srpt_aging A (>= 0).  Returns (schedule, srpt_aging)."""
    name, sep, aging = spec.partition("/")
    if name not in ("fifo", "fair", "srpt") or (sep and name != "srpt"):
        raise ValueError(f"unknown schedule {spec!r}: fifo, fair, srpt or srpt/AGING")
    a = float(aging) if sep else 0.0
    if not a >= 0.0:
        raise ValueError(f"negative srpt aging in {spec!r}")
    return name, a


def serving_study(ctx, n_requests: int = 1000, capacity_requests: int = 300, load: float = 0.8, seed: int = 2024,
                  schedules=("fifo",), path_slots: int = 1 << 18, log=None, rate: float | None = None,
                  srpt_reserve: float = 0.5, plain: bool = True, capacity_runs: bool = True,
                  lanes: int = 1) -> dict:
    """The serving workload's measurements on the 4 resident scenes (50k / 100k / 250k / 500k
    Gaussians, seeds 1-4):
      offline capacity   the first `capacity_requests` requests of the seeded stream all at t = 0
                         through one vp_render per request (the offline engine, back to back);
      served capacity    the same requests at t = 0 through the server (each schedule);
      latency            all `n_requests` with Poisson arrivals at `load` x the offline capacity,
                         served (each schedule) and through the plain per-request loop, on the same
                         arrivals: p50 / p90 / p99 / max of arrival-to-completion wall time.
    A schedule "srpt/A" is SRPT with srpt_aging A.
    `rate` (requests/s) fixes the arrival rate instead, so runs compare on identical arrivals;
    `capacity_runs` / `plain` switch those runs off.  Returns the figures as a dict."""
    from . import scenes
    gs, sigma, env_img = scenes.serving_scenes()
    scs = [Scene(ctx, g, sigma) for g in gs]
    env = Environment(ctx, rgb=env_img)
    envs = [env] * len(scs)

    def server(schedule):
        name, aging = schedule_spec(schedule)
        srv = Server(ctx, memory_budget_bytes=150 * 10 ** 9, schedule=name, path_slots=path_slots,
                     srpt_reserve=srpt_reserve, lanes=lanes, srpt_aging=aging)
        for sc in scs:
            srv.add_scene(sc, env)
        return srv

    def summary(r):
        lat = sorted(r["latency_s"])
        return {"p50_s": r["p50_s"], "p90_s": percentile(lat, 90), "p99_s": r["p99_s"], "max_s": lat[-1],
                "mpaths_per_s": r["mpaths_per_s"], "makespan_s": r["makespan_s"]}

    def emit(d):
        if log:
            log(d)

    base = make_trace(seed, n_requests, rate=1.0, n_scenes=len(scs))
    mean_paths = sum(r.paths for r in base) / len(base)
    burst = capacity(base[:capacity_requests])
    # warm-up: a few requests through both loops (first-use allocations, graph capture)
    w = server("fifo")
    run_trace(w, burst[:8])
    w.close()
    run_trace_plain(scs, envs, burst[:8])
    out = {"requests": n_requests, "capacity_requests": capacity_requests, "load": load,
           "mean_paths_per_request": mean_paths, "path_slots": path_slots, "srpt_reserve": srpt_reserve,
           "lanes": lanes}
    out["served_capacity"] = {}
    if capacity_runs:
        pl = run_trace_plain(scs, envs, burst)
        out["offline_mpaths_per_s"] = pl["mpaths_per_s"]
        emit({"run": "offline capacity (plain per-request loop, all at t = 0)", **summary(pl)})
    for sched in (schedules if capacity_runs else ()):
        srv = server(sched)
        r = run_trace(srv, burst)
        st = srv.stats()
        srv.close()
        out["served_capacity"][sched] = {"mpaths_per_s": r["mpaths_per_s"],
                                         "fraction_of_offline": r["mpaths_per_s"] / pl["mpaths_per_s"],
                                         "device_busy": st["device_ms"] / 1e3 / r["makespan_s"]}
        emit({"run": f"served capacity ({sched}, all at t = 0)", **summary(r), "device_s": st["device_ms"] / 1e3})
    if rate is None:
        rate = load * out["offline_mpaths_per_s"] * 1e6 / mean_paths
    out["arrival_rate_per_s"] = rate
    trace = make_trace(seed, n_requests, rate=rate, n_scenes=len(scs))
    out["served"] = {}
    for sched in schedules:
        srv = server(sched)
        r = run_trace(srv, trace)
        st = srv.stats()
        srv.close()
        out["served"][sched] = {**summary(r), "device_s": st["device_ms"] / 1e3, "iterations": st["iterations"]}
        emit({"run": f"served ({sched}) at {load:.0%} of offline capacity", **out["served"][sched]})
    if plain:
        pr = run_trace_plain(scs, envs, trace)
        out["plain"] = {**summary(pr), "busy_s": pr["busy_s"]}
        emit({"run": f"plain per-request loop at {load:.0%} of offline capacity", **out["plain"]})
    for sc in scs:
        sc.close()
    env.close()
    return out


def main(argv=None) -> None:
    """The serving study end to end (serving_study), one JSON line per run and a summary line."""
    import argparse
    import json
    from .api import Context
    ap = argparse.ArgumentParser(prog="python -m volprim_b200.serving")
    ap.add_argument("--requests", type=int, default=1000)
    ap.add_argument("--capacity-requests", type=int, default=300)
    ap.add_argument("--load", type=float, default=0.8)
    ap.add_argument("--schedules", default="fifo", help="comma-separated: fifo, fair, srpt, srpt/AGING")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--slots", type=int, default=1 << 18)
    ap.add_argument("--rate", type=float, default=None, help="fixed arrival rate (requests/s)")
    ap.add_argument("--srpt-reserve", type=float, default=0.5)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-capacity", action="store_true")
    ap.add_argument("--lanes", type=int, default=1)
    a = ap.parse_args(argv)
    ctx = Context(a.device)
    res = serving_study(ctx, a.requests, a.capacity_requests, a.load, a.seed, tuple(a.schedules.split(",")),
                        a.slots, log=lambda d: print(json.dumps(d), flush=True), rate=a.rate,
                        srpt_reserve=a.srpt_reserve, plain=not a.no_plain, capacity_runs=not a.no_capacity,
                        lanes=a.lanes)
    print(json.dumps({"run": "summary", **res}), flush=True)
    ctx.close()


if __name__ == "__main__":
    main()
