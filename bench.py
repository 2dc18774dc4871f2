"""Benchmark of the B200 path-tracing core: Mrays/s on the 1920x1080, 4 spp,
depth 8 workload (64 BLAS of 2k-64k triangles, 1024 instances, Lambertian +
20 % mirror; seeded synthetic scene), one JSON line on rank 0.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

A step is one frame: camera rays for every pixel and sample, then per bounce a
closest-hit trace, shading, and a shadow-ray trace, then accumulation.  The
device-timed `value` counts closest + shadow rays (the reference's counting,
rend.c:3154/3264) over the K frames with inputs resident on the device; `e2e`
runs the same frames through the C ABI as a frame loop does for a changing
scene (upload of the TLAS and instances from host memory, render, ARGB8
image back to pinned host memory).  With --gpus N under torchrun every rank
renders its own replica of the frame (the path does not shard across GPUs
in a way that needs an exchange): value = all rays / max rank time.

The reference arm (--impl reference) times the reference renderer's own CPU
traversal (intersect_tlas / intersect_any_tlas compiled from its sources)
inside the CPU restatement of the path tracer, on all host cores, on a
bounded band of rows of the same frame.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(family=2, seed=1, width=1920, height=1080, spp=4, depth=8)
L2_BYTES = 126 * 1024 * 1024


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--width", type=int, default=WORKLOAD["width"])
    p.add_argument("--height", type=int, default=WORKLOAD["height"])
    p.add_argument("--spp", type=int, default=WORKLOAD["spp"])
    p.add_argument("--depth", type=int, default=WORKLOAD["depth"])
    p.add_argument("--blas", type=int, default=0,
                   help="BLAS count (0 = the workload's 64)")
    p.add_argument("--ref-blas", action="store_true",
                   help="trace the reference's BVH8 BLASes converted node "
                   "for node instead of the library's own build")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--sort", type=int, default=0,
                   help="1: reorder each bounce's rays before tracing")
    p.add_argument("--fuse", type=int, default=0,
                   help="1: shadow rays traced with the next bounce's "
                        "closest hits, 2: separate launches, 0: default")
    p.add_argument("--update-levels", action="store_true",
                   help="e2e frames rebuild the TLAS level by level "
                   "(RENDGPU_UPDATE_LEVELS) instead of the library's "
                   "choice (the collapsed one-CTA build up to 2048 "
                   "instances)")
    p.add_argument("--queue", type=int, default=0,
                   help="camera slots per wave (0 = the library's default: "
                   "two concurrent half-frame waves)")
    p.add_argument("--block", type=int, default=0,
                   help="trace block size (0 = library default)")
    p.add_argument("--sched", type=int, default=0,
                   help="traversal schedule (0 = library default)")
    p.add_argument("--count", action="store_true",
                   help="one extra untimed frame counting node visits and "
                        "triangle tests per closest-hit ray")
    p.add_argument("--no-nrc", action="store_true",
                   help="skip the radiance-cache equal-time evaluation")
    p.add_argument("--nrc-width", type=int, default=1920)
    p.add_argument("--nrc-height", type=int, default=1080)
    p.add_argument("--nrc-frames", type=int, default=64)
    p.add_argument("--nrc-ref-spp", type=int, default=4096,
                   help="samples per pixel of the plain reference image")
    p.add_argument("--cpu-seconds", type=float, default=15.0,
                   help="target CPU time of the bounded CPU sample")
    p.add_argument("--no-batch", action="store_true",
                   help="skip the 16-scene batched workload")
    p.add_argument("--batch-frames", type=int, default=3)
    p.add_argument("--no-stress", action="store_true",
                   help="skip the 3840x2160 depth-16 stress workload")
    p.add_argument("--stress-frames", type=int, default=2)
    p.add_argument("--stress-eval-width", type=int, default=960)
    p.add_argument("--stress-eval-height", type=int, default=540)
    p.add_argument("--stress-ref-spp", type=int, default=4096)
    p.add_argument("--update-reps", type=int, default=10,
                   help="device-side scene updates timed on the stress "
                        "scene")
    p.add_argument("--stress-nrc-frames", type=int, default=32)
    return p.parse_args()


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=120))
    return world, rank, local


def allreduce(x, op):
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return x
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def job_rate(units, ms, world):
    """Whole-job rate of N replicas: all ranks' units over the slowest
    rank's device time (units per ms; collective on every rank).  Returns
    (rate, slowest ms, all units)."""
    import torch
    ms_max = allreduce(ms, torch.distributed.ReduceOp.MAX) if world > 1 \
        else ms
    units_all = allreduce(units, torch.distributed.ReduceOp.SUM) \
        if world > 1 else units
    return units_all / ms_max, ms_max, units_all


def barrier():
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def config_of(a, world):
    return {"workload": "scale: 64 BLAS (displaced spheres / triangle soups, "
            "2k-64k tris log-uniform), 1024 instances, Lambertian + 20%% "
            "mirror, ground + quad light; %dx%d, %d spp, max depth %d"
            % (a.width, a.height, a.spp, a.depth),
            "scene_seed": WORKLOAD["seed"], "width": a.width,
            "height": a.height, "spp": a.spp, "max_depth": a.depth,
            "blas": a.blas or 64, "instances": 1024,
            "parallelism": "replicas x%d" % world,
            "l2": "flushed between frames (256 MiB write), frames timed "
                  "individually with CUDA events on the library stream"}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_from_profile():
    """dram bytes per closest-hit launch from the committed ncu summary
    (a line `trace_dram_bytes_per_ray: X`), scaled by rays per launch."""
    path = os.path.join(ROOT, "profiles", "k_trace_scale.md")
    try:
        for line in open(path):
            if line.startswith("trace_dram_bytes_per_ray:"):
                return float(line.split(":")[1])
    except Exception:
        pass
    return None


class Clocks:
    """nvidia-smi sampling (every 100 ms, timestamped) started before the
    warm-up, so that it runs through the timed region; stop() keeps the
    samples taken between mark_start() and mark_end()."""
    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,"
         "clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None
        self.t0 = self.t1 = None
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None

    def mark_start(self):
        import datetime
        self.t0 = datetime.datetime.now()

    def mark_end(self):
        import datetime
        self.t1 = datetime.datetime.now()

    def stop(self):
        import datetime
        if not self.p:
            return None
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except Exception:
            self.p.kill()
            out = ""
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        rows = []
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(f[0], "%Y/%m/%d %H:%M:%S.%f")
                rows.append((ts, float(f[2]), float(f[3]), f[6:10]))
            except ValueError:
                continue
        if not rows:
            return None
        inside = [r for r in rows if self.t0 and self.t1 and
                  self.t0 <= r[0] <= self.t1]
        scope = "timed region"
        if not inside:
            # a timed region shorter than the sampling period: the samples
            # nearest to it
            mid = self.t0 + (self.t1 - self.t0) / 2 if self.t0 and self.t1 \
                else rows[-1][0]
            inside = sorted(rows, key=lambda r: abs((r[0] - mid)
                                                   .total_seconds()))[:2]
            scope = "nearest to the timed region"
        reasons = set()
        for r in inside:
            for n, v in zip(names, r[3]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(r[1] for r in inside),
                "sm_max_mhz": max(r[2] for r in inside),
                "reasons": sorted(reasons), "samples": len(inside),
                "scope": scope}


def cpu_baseline(a, rd, lights, area, budget_s):
    """Reference traversal (compiled from its sources) in the CPU path
    tracer, all host cores, on a band of rows of the same frame; plus the
    reference algorithm's visit counts (restated traversal) for the
    roofline's bytes per ray."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    cores = ol.ncpu()
    W, H = a.width, a.height
    use_ref = ol.ref() is not None
    # calibrate on 4 rows, then size the band to the time budget
    t0 = time.perf_counter()
    _, r0 = ol.orc_render(rd, lights, area, a.depth, seed=1,
                          window=(0, H // 2, W, H // 2 + 4), use_ref=use_ref)
    dt = time.perf_counter() - t0
    rows = max(4, min(H, int(4 * budget_s / max(dt, 1e-3))))
    y0 = max(0, H // 2 - rows // 2)
    t0 = time.perf_counter()
    _, rays = ol.orc_render(rd, lights, area, a.depth, seed=1,
                            window=(0, y0, W, y0 + rows), use_ref=use_ref)
    dt = time.perf_counter() - t0
    # visit counts of the reference algorithm on ~1% of the rows, spread
    # evenly over the frame
    cnt = ol.Counts()
    crays = 0
    for y in range(H // 200, H, max(1, H // 100)):
        _, cr = ol.orc_render(rd, lights, area, a.depth, seed=1,
                              window=(0, y, W, y + 1), counts=cnt)
        crays += cr
    # counts cover closest-hit rays only: shadow rays of the sample are
    # part of crays, so divide by the closest-hit share measured on the GPU
    return {"value": rays / dt / 1e6, "unit": "Mrays/s", "cores": cores,
            "kind": "reference" if use_ref else "port",
            "sample": "rows %d..%d of the %dx%d frame (%d spp, depth %d): "
                      "%d rays in %.1f s; reference intersect_tlas/"
                      "intersect_any_tlas inside the restated path tracer"
                      % (y0, y0 + rows, W, H, a.spp, a.depth, rays, dt),
            "_counts": (cnt.nodes, cnt.leaves, cnt.insts, crays)}


def _elapsed(ev):
    return sum(s.elapsed_time(e) for s, e in ev)


def batch_eval(a, dev, flush):
    """The batched uneven workload: 16 seeded scenes of the small family
    (one icosphere BLAS of 1k-1M triangles log-uniform x4 + ground + quad
    light; resolution, spp and depth drawn per scene) rendered as one
    batch (one captured launch sequence per frame over shared queues,
    launch parameters autotuned), then each scene alone."""
    import torch
    from nodebleed_b200 import api
    t0 = time.perf_counter()
    scenes = [api.Scene(api.SCENE_BATCH, 1, i) for i in range(16)]
    rds = [api.RenderData(sc) for sc in scenes]
    depths = [sc.settings()["depth"] for sc in scenes]
    host_s = time.perf_counter() - t0
    b = api.BatchRenderer(rds, max_depth=depths, seed=1, timing=True,
                          device=dev).upload()
    t0 = time.perf_counter()
    best, log = b.autotune(frames=1)
    tune_s = time.perf_counter() - t0
    stream = torch.cuda.ExternalStream(b.stream(), device=dev)
    b.frame()
    torch.cuda.synchronize()
    ev, per_rays, tot_rays, launches = [], [0] * 16, 0, 0
    for _ in range(a.batch_frames):
        with torch.cuda.stream(stream):
            flush.zero_()
            s, e = torch.cuda.Event(enable_timing=True), \
                torch.cuda.Event(enable_timing=True)
            s.record(stream)
        tot_rays += b.frame()
        with torch.cuda.stream(stream):
            e.record(stream)
        ev.append((s, e))
        tot, per = b.stats()
        launches = tot["launches"]
        for i, p in enumerate(per):
            per_rays[i] += p["closest_rays"] + p["shadow_rays"]
    torch.cuda.synchronize()
    ms = _elapsed(ev)
    b.close()
    rows, alone_ms = [], 0.0
    for i, (sc, rd) in enumerate(zip(scenes, rds)):
        gr = api.GpuRenderer(rd, max_depth=depths[i], seed=1, timing=True,
                             device=dev, graph=True).upload()
        st_ = torch.cuda.ExternalStream(gr.stream(), device=dev)
        gr.frame()
        ev1, r1 = [], 0
        for _ in range(a.batch_frames):
            with torch.cuda.stream(st_):
                flush.zero_()
                s, e = torch.cuda.Event(enable_timing=True), \
                    torch.cuda.Event(enable_timing=True)
                s.record(st_)
            r1 += gr.frame()
            with torch.cuda.stream(st_):
                e.record(st_)
            ev1.append((s, e))
        torch.cuda.synchronize()
        m1 = _elapsed(ev1)
        alone_ms += m1
        gr.close()
        cfg = sc.settings()
        rows.append({"scene": i, "tris": sc.tris,
                     "res": [cfg["width"], cfg["height"]],
                     "spp": cfg["spp"], "depth": cfg["depth"],
                     "rays_per_frame": per_rays[i] / a.batch_frames,
                     "mrays_s_share_in_batch": per_rays[i] / ms / 1e3,
                     "mrays_s_alone": r1 / m1 / 1e3,
                     "ms_alone": m1 / a.batch_frames})
    return {"workload": "16 scenes of the small family (seed 1, scene "
                        "index 0..15): 1k-1M tris log-uniform, resolutions "
                        "320x180..1920x1080, spp {1,4,16}, depth {4,8,12}",
            "frames": a.batch_frames,
            "aggregate_mrays_s": tot_rays / ms / 1e3,
            "ms_per_frame": ms / a.batch_frames,
            "alone_ms_per_frame_sum": alone_ms / a.batch_frames,
            "speedup_vs_alone": alone_ms / ms,
            "gpu_launches_per_frame": launches,
            "tuned": best, "autotune_log": log, "autotune_s": tune_s,
            "host_build_s": host_s, "scenes": rows,
            "paths_per_frame": sum(r["spp"] * r["res"][0] * r["res"][1]
                                   for r in rows),
            "unique_tris": sum(r["tris"] for r in rows)}


def update_times(a, scene, rd, gr, stream):
    """Per-frame cost of a transform change on a scene: the device path
    (rendgpu_update_instances_device: inverse, world boxes, TLAS build or
    refit, light table; CUDA events) against the host path the reference's
    frame loop runs (upd_rinsts + rend_prepdynamic restated in the host
    library, then rendgpu_upload_dynamic; wall clock)."""
    import numpy as np
    import torch
    globs = torch.from_numpy(np.ascontiguousarray(scene.globs(),
                                                  np.float32)).cuda()
    torch.cuda.synchronize()
    out = {}
    # the default level-by-level build, the one-CTA build collapsed by
    # cost (RENDGPU_UPDATE_COLLAPSE), and a refit of the default build
    for name, kw in (("device_build_collapse_ms", {"collapse": True}),
                     ("device_build_ms", {"collapse": False}),
                     ("device_refit_ms", {"refit": True,
                                          "collapse": False})):
        gr.update_instances(globs.data_ptr(), collapse=False)  # builds
        ev = []
        for _ in range(a.update_reps):
            with torch.cuda.stream(stream):
                s, e = torch.cuda.Event(enable_timing=True), \
                    torch.cuda.Event(enable_timing=True)
                s.record(stream)
            gr.update_instances(globs.data_ptr(), **kw)
            with torch.cuda.stream(stream):
                e.record(stream)
            ev.append((s, e))
        torch.cuda.synchronize()
        out[name] = _elapsed(ev) / a.update_reps
    _, _, info = gr.instances()
    out["device_tlas_nodes"], out["device_tlas_depth"] = info[0], info[1]
    t0 = time.perf_counter()
    for _ in range(max(1, a.update_reps // 5)):
        rd.update_host()
        gr.upload_dynamic()
    out["host_ms"] = (time.perf_counter() - t0) * 1e3 / \
        max(1, a.update_reps // 5)
    out["instances"] = scene.insts
    return out


def stress_eval(a, dev, flush):
    """The stress workload: 128 BLAS of 1k-200k triangles, 4096 instances
    (the reference's cap), Lambertian / GGX (roughness U[0.05,0.5]) /
    mirror thirds, 8 quad lights, 3840x2160, 1 spp, depth 16.  Plain
    wavefront throughput at full size; the reference traversal in the CPU
    path tracer on a band of rows; radiance cache against plain at equal
    device time on a reduced image (relMSE against a high-spp plain
    reference)."""
    import torch
    from nodebleed_b200 import api, nrc_eval
    t0 = time.perf_counter()
    scene = api.Scene(api.SCENE_STRESS, 1)
    rd = api.RenderData(scene)
    host_s = time.perf_counter() - t0
    cfg = scene.settings()
    W, H, depth = cfg["width"], cfg["height"], cfg["depth"]
    gr = api.GpuRenderer(rd, max_depth=depth, seed=1, timing=True,
                         device=dev, graph=True).upload()
    stream = torch.cuda.ExternalStream(gr.stream(), device=dev)
    gr.frame()
    ev, rays = [], 0
    for _ in range(a.stress_frames):
        with torch.cuda.stream(stream):
            flush.zero_()
            s, e = torch.cuda.Event(enable_timing=True), \
                torch.cuda.Event(enable_timing=True)
            s.record(stream)
        rays += gr.frame()
        with torch.cuda.stream(stream):
            e.record(stream)
        ev.append((s, e))
    torch.cuda.synchronize()
    ms = _elapsed(ev)
    st = gr.stats()
    lights, area = gr.lights()
    upd = update_times(a, scene, rd, gr, stream)
    gr.close()
    out = {"workload": "stress: 128 BLAS (1k-200k tris log-uniform), 4096 "
                       "instances, Lambertian/GGX/mirror thirds, 8 quad "
                       "lights; %dx%d, 1 spp, max depth %d" % (W, H, depth),
           "unique_tris": scene.tris, "instanced_tris": scene.inst_tris,
           "instances": scene.insts, "host_build_s": host_s,
           "mrays_s": rays / ms / 1e3,
           "samples_s": W * H * a.stress_frames / (ms / 1e3),
           "ms_per_frame": ms / a.stress_frames,
           "rays_per_frame": rays / a.stress_frames,
           "max_stack": st["max_stack"], "scene_update": upd}
    if not a.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_lib as ol
        use_ref = ol.ref() is not None
        t0 = time.perf_counter()
        _, r0 = ol.orc_render(rd, lights, area, depth, seed=1,
                              window=(0, H // 2, W, H // 2 + 2),
                              use_ref=use_ref)
        dt = time.perf_counter() - t0
        rows = max(2, min(H, int(2 * 10.0 / max(dt, 1e-3))))
        y0 = max(0, H // 2 - rows // 2)
        t0 = time.perf_counter()
        _, n = ol.orc_render(rd, lights, area, depth, seed=1,
                             window=(0, y0, W, y0 + rows), use_ref=use_ref)
        dt = time.perf_counter() - t0
        out["cpu_reference"] = {
            "mrays_s": n / dt / 1e6, "cores": ol.ncpu(),
            "kind": "reference" if use_ref else "port",
            "sample": "rows %d..%d (%d rays in %.1f s)" % (y0, y0 + rows,
                                                          n, dt)}
        out["gpu_over_cpu"] = out["mrays_s"] / out["cpu_reference"]["mrays_s"]
    t0 = time.perf_counter()
    ref = nrc_eval.reference(scene, a.stress_eval_width,
                             a.stress_eval_height, depth, a.stress_ref_spp)
    ev_ = nrc_eval.equal_time(scene, a.stress_eval_width,
                              a.stress_eval_height, depth,
                              a.stress_nrc_frames, ref, batch=True)
    out["equal_time"] = {"width": a.stress_eval_width,
                         "height": a.stress_eval_height,
                         "reference_spp": a.stress_ref_spp,
                         "nrc": {k: ev_["nrc"][k] for k in
                                 ("frames", "ms", "relmse", "rays",
                                  "batched")},
                         "plain": ev_["plain"],
                         "ratio_plain_over_nrc":
                             ev_["ratio_plain_over_nrc"],
                         "wall_s": time.perf_counter() - t0}
    rd.close()
    return out


def run_ours(a):
    import numpy as np
    import torch
    from nodebleed_b200 import api

    world, rank, local = dist_setup()
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    scene = api.Scene(WORKLOAD["family"], WORKLOAD["seed"], a.blas)
    rd = api.RenderData(scene, a.width, a.height, a.spp)
    gr = api.GpuRenderer(rd, max_depth=a.depth, seed=1 + rank, timing=True,
                         device=dev, sched=a.sched,
                         ref_blas=a.ref_blas).upload()
    if a.sort or a.block or a.fuse or a.queue:
        gr.set_tune(sort=a.sort, block=a.block, fuse=a.fuse, queue=a.queue)
    stream = torch.cuda.ExternalStream(gr.stream(), device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    lights, area = gr.lights()

    clocks = Clocks(dev)
    for _ in range(a.warmup):
        gr.frame()
    barrier()
    torch.cuda.synchronize()
    clocks.mark_start()
    ev = []
    rays = closest = 0
    trace_ms = shadow_ms = 0.0
    launches = trace_launches = 0
    for _ in range(a.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            s, e = torch.cuda.Event(enable_timing=True), \
                torch.cuda.Event(enable_timing=True)
            s.record(stream)
        n = gr.frame()
        with torch.cuda.stream(stream):
            e.record(stream)
        st = gr.stats()
        rays += n
        closest += st["closest_rays"]
        trace_ms += st["ms_trace"]
        shadow_ms += st["ms_shadow"]
        launches += st["launches"]
        trace_launches += st["trace_launches"]
        ev.append((s, e))
    torch.cuda.synchronize()
    clocks.mark_end()
    cl = clocks.stop()
    barrier()
    ms = sum(s.elapsed_time(e) for s, e in ev)
    rate, ms_max, rays_all = job_rate(rays, ms, world)
    samples_all = a.width * a.height * a.spp * a.steps * world
    value = rate / 1e3  # rays per ms -> Mrays/s

    # end to end through the C ABI with host buffers
    e2e = None
    if not a.no_e2e:
        pinned = torch.empty(a.width * a.height, dtype=torch.int32,
                             pin_memory=True)
        rd.buf = pinned.numpy().view(np.uint32)
        rd.rd.buf = pinned.data_ptr()
        h2d = d2h = 0
        e2e_rays = 0
        # the frame loop of a moving scene: new object->world matrices from
        # host memory every frame; the device inverts them, rebuilds the
        # TLAS and the light table (rendgpu_update_instances)
        globs = np.ascontiguousarray(scene.globs(), np.float32)
        barrier()
        torch.cuda.synchronize()
        parts = [0.0, 0.0, 0.0]
        t0 = time.perf_counter()
        for _ in range(a.steps):
            t1 = time.perf_counter()
            gr.update_instances(globs, tight=True,
                                collapse=False if a.update_levels else None)
            h2d += gr.stats()["h2d_bytes"]
            t2 = time.perf_counter()
            e2e_rays += gr.frame()
            t3 = time.perf_counter()
            gr.readback(2)
            d2h += gr.stats()["d2h_bytes"]
            t4 = time.perf_counter()
            parts[0] += t2 - t1
            parts[1] += t3 - t2
            parts[2] += t4 - t3
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        # the roofline frames below use the uploaded (host-built) TLAS, as
        # the timed frames did
        gr.upload_dynamic()
        e2e_rate, _, _ = job_rate(e2e_rays, dt, world)
        e2e = {"value": e2e_rate / 1e6, "unit": "Mrays/s",
               "h2d_bytes_per_step": h2d // a.steps,
               "d2h_bytes_per_step": d2h // a.steps,
               "timing": "wall clock around the scene update from host "
                         "matrices (device inverse, TLAS build and light "
                         "table) + render + readback of the ARGB8 image "
                         "(pinned host)",
               "ms_upload_render_readback": [1e3 * x / a.steps
                                             for x in parts]}

    # the roofline's kernel alone: closest-hit launches timed in frames
    # whose shadow rays go to separate launches
    sep_trace_ms = sep_closest = sep_launches = 0
    if rank == 0 and world == 1:
        # separate shadow launches and one wave of all paths, so that each
        # closest-hit launch runs alone on the GPU
        tune = gr.get_tune()
        gr.set_tune(**{k: tune[k] for k in ("block", "stack", "sched",
                                             "sort")}, fuse=2,
                    queue=0x7fffffff)
        gr.frame()
        for _ in range(2):
            with torch.cuda.stream(stream):
                flush.zero_()
            gr.frame()
            st2 = gr.stats()
            sep_trace_ms += st2["ms_trace"]
            sep_closest += st2["closest_rays"]
            sep_launches += st2["trace_launches"]
        gr.set_tune(**{k: tune[k] for k in ("block", "stack", "queue",
                                             "sched", "sort", "fuse")})

    visits = None
    if a.count:
        # one context per rdata: the counting context replaces the timed one
        gr.close()
        gc = api.GpuRenderer(rd, max_depth=a.depth, seed=1 + rank,
                             count=True, device=dev, sched=a.sched,
                             ref_blas=a.ref_blas).upload()
        gc.frame()
        sc = gc.stats()
        visits = {"nodes_per_ray": sc["node_visits"] / sc["closest_rays"],
                  "tri_tests_per_ray": sc["tri_tests"] / sc["closest_rays"]}
        gc.close()

    nrc = None
    if rank == 0 and world == 1 and not a.no_nrc:
        # radiance cache vs plain at equal device time, 1 spp per frame,
        # both against a high-spp plain reference (relMSE in FP64 on the
        # device); the same scene as the throughput workload
        from nodebleed_b200 import nrc_eval
        t0 = time.perf_counter()
        ref = nrc_eval.reference(scene, a.nrc_width, a.nrc_height, a.depth,
                                 a.nrc_ref_spp)
        nrc = nrc_eval.equal_time(scene, a.nrc_width, a.nrc_height, a.depth,
                                  a.nrc_frames, ref)
        nrc["config"] = {"width": a.nrc_width, "height": a.nrc_height,
                         "spp_per_frame": 1, "depth": a.depth,
                         "reference_spp": a.nrc_ref_spp,
                         "warmup_frames": 1, "self_train_bounce": 3,
                         "train_paths_per_frame": 65536,
                         "adam_steps_per_frame": 6, "adam_lr": 1e-2}
        nrc["wall_s"] = time.perf_counter() - t0

    batch = None
    if rank == 0 and world == 1 and not a.no_batch:
        gr.close()
        batch = batch_eval(a, dev, flush)

    stress = None
    if rank == 0 and world == 1 and not a.no_stress:
        gr.close()
        stress = stress_eval(a, dev, flush)

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline(a, rd, lights, area, a.cpu_seconds)

    out = None
    if rank == 0:
        peak, peak_kind = measured_peaks()
        roof = None
        if cpu is not None:
            nodes, leaves, insts, crays = cpu.pop("_counts")
            # closest-hit rays of the counted sample: the GPU's closest
            # share applied to the sample's ray count
            share = closest / max(rays, 1)
            csample = max(crays * share, 1.0)
            b_ray = (256.0 * nodes + 192.0 * leaves + 64.0 * insts) / \
                csample + 48.0
            per_launch_rays = sep_closest / max(sep_launches, 1)
            launch_ms = sep_trace_ms / max(sep_launches, 1)
            achieved = per_launch_rays * b_ray / (launch_ms / 1e3) / 1e9
            traffic = traffic_from_profile()
            roof = {"bound": "hbm", "achieved": achieved, "peak": peak,
                    "unit": "GB/s", "frac": achieved / peak,
                    "peak_source": peak_kind,
                    "kernel": "k_trace (closest hit; timed in frames "
                              "with separate shadow launches)",
                    "bytes_per_ray": b_ray,
                    "visits_per_ray": [nodes / csample, leaves / csample,
                                       insts / csample],
                    "traffic": traffic * per_launch_rays if traffic else None,
                    "launch_ms": launch_ms, "rays_per_launch": per_launch_rays}
        out = {"metric": "Mrays/s", "value": value, "unit": "Mrays/s",
               "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
               "ms_per_step": ms_max / a.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f32",
               "data": "synthetic (seeded procedural scene)",
               "config": config_of(a, world),
               "samples_per_s": samples_all / (ms_max / 1e3),
               "rays_per_frame": rays / a.steps,
               "closest_rays_per_frame": closest / a.steps,
               "rays_per_bounce": {"closest": st["bounce_closest"][:a.depth],
                                   "shadow": st["bounce_shadow"][:a.depth]},
               "ms_trace_per_frame": trace_ms / a.steps,
               "ms_shadow_per_frame": shadow_ms / a.steps,
               "gpu_launches": launches, "e2e": e2e, "roofline": roof,
               "gpu_visits": visits, "nrc": nrc, "batch": batch,
               "stress": stress,
               "cpu_baseline": cpu, "clocks": cl,
               "scene": {"unique_tris": scene.tris,
                         "instanced_tris": scene.inst_tris,
                         "instances": scene.insts}}
        print(json.dumps(out), flush=True)
    gr.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return out


def run_reference(a):
    # rank 0 alone times the CPU reference; other ranks exit without work
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if int(os.environ.get("RANK", "0")) != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    from nodebleed_b200 import api
    scene = api.Scene(WORKLOAD["family"], WORKLOAD["seed"], a.blas)
    rd = api.RenderData(scene, a.width, a.height, a.spp)
    # light table: the same emitters the GPU arm samples (FP64, numpy)
    from test_oracle import _lights_numpy
    lights, area = _lights_numpy(rd)
    use_ref = ol.ref() is not None
    W, H = a.width, a.height
    t0 = time.perf_counter()
    ol.orc_render(rd, lights, area, a.depth, seed=1,
                  window=(0, H // 2, W, H // 2 + 2), use_ref=use_ref)
    dt = time.perf_counter() - t0
    per_step = max(10.0, 60.0 / max(a.steps + a.warmup, 1))
    rows = max(2, min(H, int(2 * per_step / max(dt, 1e-3))))
    y0 = max(0, H // 2 - rows // 2)
    for _ in range(a.warmup):
        ol.orc_render(rd, lights, area, a.depth, seed=1,
                      window=(0, y0, W, y0 + max(2, rows // 8)),
                      use_ref=use_ref)
    tot_rays, tot_s = 0, 0.0
    for k in range(a.steps):
        t0 = time.perf_counter()
        _, n = ol.orc_render(rd, lights, area, a.depth, seed=1 + k,
                             window=(0, y0, W, y0 + rows), use_ref=use_ref)
        tot_s += time.perf_counter() - t0
        tot_rays += n
    v = tot_rays / tot_s / 1e6
    sample = ("rows %d..%d of the %dx%d frame per step (%d spp, depth %d); "
              "reference intersect_tlas/intersect_any_tlas inside the "
              "restated path tracer" % (y0, y0 + rows, W, H, a.spp, a.depth))
    out = {"impl": "reference", "metric": "Mrays/s", "value": v,
           "unit": "Mrays/s", "n_gpus": world, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": tot_s / a.steps * 1e3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f32", "data": "synthetic (seeded procedural scene)",
           "config": config_of(a, world),
           "cpu_baseline": {"value": v, "unit": "Mrays/s",
                            "cores": ol.ncpu(),
                            "kind": "reference" if use_ref else "port",
                            "sample": sample},
           "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
