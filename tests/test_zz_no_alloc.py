"""The allocation-free trace entry point (rendgpu_trace_rays_device_noalloc)
against the regular device entry point (rendgpu_trace_rays_device).

Callers that may not have the library allocate device memory mid-run (an
application that owns all device memory through its own arena, or a frame
loop that cannot absorb the device synchronisation a cudaMalloc/cudaFree can
imply) use the no-alloc form; its scratch is one fixed static device array.
The two must agree bit for bit, also on a second call that reuses the array
left over from the first.  This file is collected last so that a failure
here stops a `-x` run only after every other test has run.
"""

import numpy as np
import pytest

from nodebleed_b200 import api
import oracle_lib as ol

pytestmark = pytest.mark.gpu

MAX_RAYS = 1 << 18


def _device(arr):
    import torch
    return torch.from_numpy(np.ascontiguousarray(arr).view(np.uint8)).cuda()


def _trace(gr, fn, d_rays, n):
    import torch
    out = torch.full((n * 16,), 0xAB, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    rc = fn(gr.ptr, d_rays.data_ptr(), n, out.data_ptr())
    assert rc == 0, gr.g.rendgpu_strerror(gr.ptr)
    assert gr.g.rendgpu_sync(gr.ptr) == 0
    return out.cpu().numpy().view(api.HIT_DTYPE)


def test_noalloc_matches_device_entry_point(gpu):
    scene = api.Scene(api.SCENE_SMALL, 1)
    rd = api.RenderData(scene)
    gr = api.GpuRenderer(rd).upload()
    g = gr.g
    sets = [np.concatenate([ol.random_rays(rd, 60000, seed=5),
                            ol.camera_rays(rd)[::5]]),
            ol.random_rays(rd, 20000, seed=6)]
    for rays in sets:  # two calls in a row, different sizes
        n = len(rays)
        assert n <= MAX_RAYS
        d_rays = _device(rays)
        ref = _trace(gr, g.rendgpu_trace_rays_device, d_rays, n)
        got = _trace(gr, g.rendgpu_trace_rays_device_noalloc, d_rays, n)
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
        assert (got["t"] < ol.FLT_MAX).sum() > n // 10
    gr.close()


def test_noalloc_full_array_and_error_report(gpu):
    """A batch of exactly the maximum fills the array to its last hit
    record; rays the device abandons (an 8-entry stack forced on a deep
    scene) come back as misses and are reported by rendgpu_sync."""
    scene = api.Scene(api.SCENE_SCALE, 3, 8)
    rd = api.RenderData(scene)
    gr = api.GpuRenderer(rd).upload()
    g = gr.g
    rays = ol.random_rays(rd, MAX_RAYS, seed=8)
    d_rays = _device(rays)
    ref = _trace(gr, g.rendgpu_trace_rays_device, d_rays, MAX_RAYS)
    got = _trace(gr, g.rendgpu_trace_rays_device_noalloc, d_rays, MAX_RAYS)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    gr.set_tune(stack=8, force=1)
    import torch
    out = torch.zeros(MAX_RAYS * 16, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    assert g.rendgpu_trace_rays_device_noalloc(
        gr.ptr, d_rays.data_ptr(), MAX_RAYS, out.data_ptr()) == 0
    assert g.rendgpu_sync(gr.ptr) == -6  # RENDGPU_EDEVICE
    assert gr.stats()["device_errors"] > 0
    lost = out.cpu().numpy().view(api.HIT_DTYPE)
    diff = lost.view(np.uint32).reshape(-1, 4) != \
        ref.view(np.uint32).reshape(-1, 4)
    assert (lost["t"][diff.any(axis=1)] == ol.FLT_MAX).all()
    gr.set_tune()
    assert g.rendgpu_sync(gr.ptr) == 0
    gr.close()


def test_noalloc_rejects_oversized_batch(gpu):
    scene = api.Scene(api.SCENE_TINY, 1)
    rd = api.RenderData(scene)
    gr = api.GpuRenderer(rd).upload()
    rc = gr.g.rendgpu_trace_rays_device_noalloc(gr.ptr, 16, MAX_RAYS + 1, 16)
    assert rc == -4  # RENDGPU_ELIMIT, before any device work
    assert b"exceeds" in gr.g.rendgpu_strerror(gr.ptr)
    gr.close()
