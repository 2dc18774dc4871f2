"""Equal-time comparison of the radiance-cache renderer with the plain
wavefront path tracer, both against a high-spp plain reference; relMSE is
reduced on the device in FP64 (rendgpu_relmse_device)."""

import numpy as np

from . import api


def reference(scene, w, h, depth, spp, seed=99, spp_per_frame=16):
    """Converged plain image (H, W, 3) of `spp` samples per pixel."""
    rd = api.RenderData(scene, w, h, spp_per_frame)
    gr = api.GpuRenderer(rd, max_depth=depth, seed=seed).upload()
    for _ in range(max(1, spp // spp_per_frame)):
        gr.frame()
    gr.readback(1)
    img = rd.acc() / float(rd.rd.samples)
    gr.close()
    rd.close()
    return img.astype(np.float32)


def relmse_host(acc, samples, ref):
    """The relMSE of rendgpu_relmse_device computed on the host in FP64:
    mean of (x - r)^2 / (r^2 + 0.01) with x = acc * (1 / samples as FP32)."""
    inv = np.float32(1.0) / np.float32(samples)
    x = np.asarray(acc, np.float32).astype(np.float64) * np.float64(inv)
    r = np.asarray(ref, np.float32).astype(np.float64)
    return float(np.mean((x - r) ** 2 / (r * r + 0.01)))


def _load_cache_kernels(depth):
    """Two radiance-cache frames of a tiny scene on a throwaway context, so
    the first launch of each cache kernel (module loading) is not counted
    in the timed frames."""
    sc = api.Scene(api.SCENE_TINY, 1)
    rd = api.RenderData(sc)
    g = api.GpuRenderer(rd, max_depth=depth, mode=api.MODE_NRC,
                        nrc_warmup=1).upload()
    g.frame()
    g.frame()
    g.close()
    rd.close()


def equal_time(scene, w, h, depth, frames, ref, seed=1, **nrc_kw):
    """NRC for `frames` frames of 1 spp, then plain 1-spp frames until the
    same device time; relMSE of both accumulated images against `ref`.
    nrc_kw go to the cache renderer (nrc_warmup, nrc_end, nrc_lr)."""
    import torch
    batch = nrc_kw.pop("batch", False)
    _load_cache_kernels(depth)
    ref_dev = torch.from_numpy(np.ascontiguousarray(ref, np.float32)).cuda()
    out = {}
    rd = api.RenderData(scene, w, h, 1)
    if batch:
        # the cache frames through the batch API (one launch sequence over
        # shared queues, as a batch of scenes runs them)
        gn = api.BatchRenderer([rd], max_depth=depth, mode=api.MODE_NRC,
                               seed=seed, timing=True,
                               nrc_grid=nrc_kw.get("nrc_grid", True)).upload()

        def stats():
            return gn.stats()[0]

        def err():
            gn.readback(1)
            return relmse_host(rd.acc(), rd.rd.samples, ref)
    else:
        gn = api.GpuRenderer(rd, max_depth=depth, mode=api.MODE_NRC,
                             seed=seed, timing=True, **nrc_kw).upload()
        stats = gn.stats

        def err():
            return gn.relmse(ref_dev.data_ptr())
    t_nrc, rays_nrc, curve = 0.0, 0, []
    for f in range(frames):
        rays_nrc += gn.frame()
        st = stats()
        t_nrc += st["ms_frame"]
        if f in (0, frames // 4, frames // 2, frames - 1):
            curve.append((f + 1, t_nrc, err()))
    out["nrc"] = {"frames": frames, "ms": t_nrc, "relmse": err(),
                  "rays": rays_nrc, "queries_last": st["nrc_queries"],
                  "records_last": st["nrc_records"],
                  "ms_cache_last": st["ms_nrc"], "curve": curve,
                  "batched": bool(batch)}
    gn.close()
    rd.close()
    rd = api.RenderData(scene, w, h, 1)
    gp = api.GpuRenderer(rd, max_depth=depth, mode=api.MODE_PATH, seed=seed,
                         timing=True).upload()
    t_plain, fp, rays_plain = 0.0, 0, 0
    while t_plain < t_nrc or fp == 0:
        rays_plain += gp.frame()
        t_plain += gp.stats()["ms_frame"]
        fp += 1
    out["plain"] = {"frames": fp, "ms": t_plain,
                    "relmse": gp.relmse(ref_dev.data_ptr()),
                    "rays": rays_plain}
    gp.close()
    rd.close()
    out["ratio_plain_over_nrc"] = out["plain"]["relmse"] / \
        max(out["nrc"]["relmse"], 1e-30)
    return out


def kernel_times(n_query=700_000, n_train=16_384, reps=20, seed=3):
    """Warm CUDA-event times (us per call) of the cache's two device entry
    points on random BF16 feature rows: inference of n_query rows
    (rendgpu_nrc_infer_device) and one Adam step of n_train rows
    (rendgpu_nrc_train_device).  n_query = 700k is about the number of
    queries of a 1080p radiance-cache frame."""
    import torch
    sc = api.Scene(api.SCENE_TINY, 1)
    rd = api.RenderData(sc)
    gr = api.GpuRenderer(rd).upload()
    gr.nrc_reset(seed)
    gen = torch.Generator(device="cuda").manual_seed(seed)
    f = torch.rand((n_train, 64), device="cuda",
                   generator=gen).to(torch.bfloat16)
    t = torch.rand((n_train, 4), device="cuda", generator=gen)
    fq = torch.rand((n_query, 64), device="cuda",
                    generator=gen).to(torch.bfloat16)
    out = torch.zeros((n_query, 4), device="cuda")
    s = torch.cuda.ExternalStream(gr.stream())
    calls = {
        "train": lambda: gr._ck(gr.g.rendgpu_nrc_train_device(
            gr.ptr, f.data_ptr(), t.data_ptr(), n_train, 1, None, None),
            "nrc_train_device"),
        "infer": lambda: gr._ck(gr.g.rendgpu_nrc_infer_device(
            gr.ptr, fq.data_ptr(), n_query, out.data_ptr()),
            "nrc_infer_device")}
    res = {"n_query": n_query, "n_train": n_train}
    torch.cuda.synchronize()
    for name, fn in calls.items():
        for _ in range(3):
            fn()
        gr._ck(gr.g.rendgpu_sync(gr.ptr), "sync")
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(reps):
            fn()
        e1.record(s)
        torch.cuda.synchronize()
        res[name + "_us"] = e0.elapsed_time(e1) / reps * 1e3
    gr._ck(gr.g.rendgpu_sync(gr.ptr), "sync")
    gr.close()
    rd.close()
    return res


def cache_frames(frames=8, w=1920, h=1080, depth=8):
    """Render `frames` radiance-cache frames of the scale scene (1 spp);
    device milliseconds per frame (for launch lists and timelines)."""
    _load_cache_kernels(depth)
    scene = api.Scene(api.SCENE_SCALE, 1)
    rd = api.RenderData(scene, w, h, 1)
    g = api.GpuRenderer(rd, max_depth=depth, mode=api.MODE_NRC,
                        timing=True).upload()
    ms = []
    for _ in range(frames):
        g.frame()
        ms.append(g.stats()["ms_frame"])
    g.close()
    rd.close()
    return ms


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--kernels", action="store_true",
                    help="time the cache's inference and training calls")
    ap.add_argument("--queries", type=int, default=700_000)
    ap.add_argument("--train-rows", type=int, default=16_384)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--frames", type=int, default=0,
                    help="render this many 1080p radiance-cache frames of "
                    "the scale scene and print their device times")
    a = ap.parse_args()
    if a.kernels:
        print(json.dumps(kernel_times(a.queries, a.train_rows, a.reps)))
    elif a.frames:
        print(json.dumps({"ms_per_frame": cache_frames(a.frames)}))
    else:
        ap.print_help()
