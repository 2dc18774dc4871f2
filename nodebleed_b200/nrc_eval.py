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
    _load_cache_kernels(depth)
    ref_dev = torch.from_numpy(np.ascontiguousarray(ref, np.float32)).cuda()
    out = {}
    rd = api.RenderData(scene, w, h, 1)
    gn = api.GpuRenderer(rd, max_depth=depth, mode=api.MODE_NRC, seed=seed,
                         timing=True, **nrc_kw).upload()
    t_nrc, rays_nrc, curve = 0.0, 0, []
    for f in range(frames):
        rays_nrc += gn.frame()
        st = gn.stats()
        t_nrc += st["ms_frame"]
        if f in (0, frames // 4, frames // 2, frames - 1):
            curve.append((f + 1, t_nrc, gn.relmse(ref_dev.data_ptr())))
    out["nrc"] = {"frames": frames, "ms": t_nrc,
                  "relmse": gn.relmse(ref_dev.data_ptr()),
                  "rays": rays_nrc, "queries_last": st["nrc_queries"],
                  "records_last": st["nrc_records"],
                  "ms_cache_last": st["ms_nrc"], "curve": curve}
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
