"""Device-side scene update (rendgpu_update_instances*) against the host path
the reference's frame loop runs after a transform change (main.c:257-264):
upd_rinsts (main.c:117-157), rend_prepdynamic (rend.c:3073-3090), then the
upload of the host-built TLAS (rendgpu_upload_dynamic).

* world->object matrices and world boxes: bit-identical to the host bridge;
* light table: bit-identical to the host's;
* closest hits and any hits through the device-built (or refitted) TLAS:
  bit-identical to those through the host-built TLAS (hits do not depend on
  the tree's shape: the closest hit is the minimum over the same triangle
  tests, lowest triangle on equal t);
* whole frames: bit-identical images.
"""

import numpy as np
import pytest

from nodebleed_b200 import api
import oracle_lib as ol

pytestmark = pytest.mark.gpu


def _rotation(axis, angle):
    axis = axis / np.linalg.norm(axis)
    x, y, z = axis
    c, s = np.cos(angle), np.sin(angle)
    C = 1.0 - c
    return np.array([[c + x * x * C, x * y * C - z * s, x * z * C + y * s],
                     [y * x * C + z * s, c + y * y * C, y * z * C - x * s],
                     [z * x * C - y * s, z * y * C + x * s, c + z * z * C]])


def _move(globs, rng, angle, shift):
    """Each instance turned about a random axis through the world origin
    by up to `angle` and shifted by up to `shift`."""
    out = globs.astype(np.float64).reshape(-1, 4, 4).copy()
    for m in out:
        R = _rotation(rng.normal(size=3), rng.uniform(-angle, angle))
        m[:3, :3] = R @ m[:3, :3]
        m[:3, 3] = R @ m[:3, 3] + rng.uniform(-shift, shift, 3)
    return out.reshape(-1, 16).astype(np.float32)


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _frame(gr, rd):
    samples = rd.rd.samples
    gr.frame()
    rd.rd.samples = samples
    gr.readback(1)
    return rd.acc().copy()


def _compare(gd, gh, rd_d, rd_h, rays, what):
    xf, wb, info = gd.instances()
    assert np.array_equal(_bits(xf), _bits(rd_h.globinv())), what
    assert np.array_equal(_bits(wb), _bits(rd_h.aabbs())), what
    assert info[2] == 0 and info[0] >= 1, (what, info)
    hd, hh = gd.trace(rays), gh.trace(rays)
    assert np.array_equal(_bits(hd), _bits(hh)), what
    assert (hd["t"] < ol.FLT_MAX).mean() > 0.1
    assert np.array_equal(gd.occluded(rays), gh.occluded(rays)), what
    ld, ad = gd.lights()
    lh, ah = gh.lights()
    assert np.array_equal(_bits(ld), _bits(lh)) and ad == ah, what
    return info


def test_device_update_matches_host_path(gpu):
    scene = api.Scene(api.SCENE_SCALE, 3, 8)  # 8 BLAS, 1024 instances
    rd_d = api.RenderData(scene, 160, 90, 1)
    rd_h = api.RenderData(scene, 160, 90, 1)
    gd = api.GpuRenderer(rd_d, max_depth=4, seed=5).upload()
    rng = np.random.default_rng(11)
    rays = np.concatenate([ol.random_rays(rd_d, 60000, seed=2),
                           ol.camera_rays(rd_d)[::3]])
    globs = scene.globs()
    moved = _move(globs, rng, 0.3, 0.5)
    globs[:] = moved
    rd_h.update_host()
    gh = api.GpuRenderer(rd_h, max_depth=4, seed=5).upload()
    gd.update_instances(moved)  # host matrices, copied
    info = _compare(gd, gh, rd_d, rd_h, rays, "build")
    print(f"device TLAS: {info[0]} nodes, depth {info[1]}")
    assert np.array_equal(_bits(_frame(gd, rd_d)), _bits(_frame(gh, rd_h)))
    # tight instance boxes (every transformed vertex): smaller boxes, another
    # TLAS, the same hits
    gd.update_instances(moved, tight=True)
    _, wt, info_t = gd.instances()
    wc = rd_h.aabbs()

    def area(b):
        d = np.maximum(b[:, 3:] - b[:, :3], 0.0).astype(np.float64)
        return (d[:, 0] * d[:, 1] + d[:, 1] * d[:, 2] + d[:, 2] * d[:, 0])
    assert area(wt).sum() < area(wc).sum()
    assert info_t[2] == 0
    assert np.array_equal(_bits(gd.trace(rays)), _bits(gh.trace(rays)))
    assert np.array_equal(gd.occluded(rays), gh.occluded(rays))
    assert np.array_equal(_bits(_frame(gd, rd_d)), _bits(_frame(gh, rd_h)))
    # a small further move, refitted on the device (device matrices)
    import torch
    moved2 = _move(moved, rng, 0.02, 0.05)
    globs[:] = moved2
    rd_h.update_host()
    gh.upload_dynamic()
    d_globs = torch.from_numpy(moved2.copy()).cuda()
    torch.cuda.synchronize()
    gd.update_instances(d_globs.data_ptr(), refit=True)
    _compare(gd, gh, rd_d, rd_h, rays, "refit")
    assert np.array_equal(_bits(_frame(gd, rd_d)), _bits(_frame(gh, rd_h)))
    assert gd.g.rendgpu_sync(gd.ptr) == 0
    # wrong count: rejected before any device work
    rc = gd.g.rendgpu_update_instances_device(gd.ptr, d_globs.data_ptr(),
                                              rd_d.rd.instcnt - 1, 0)
    assert rc == -1
    # rendgpu_upload_dynamic makes the host-built TLAS current again
    gd.upload_dynamic()
    with pytest.raises(api.RendgpuError):
        gd.instances()  # world boxes only after a device-side update
    gd.close()
    gh.close()


def test_device_update_stress_scene(gpu):
    """Config 5's scene: 4096 instances, 8 lights."""
    scene = api.Scene(api.SCENE_STRESS, 1)
    rd_d = api.RenderData(scene, 192, 108, 1)
    rd_h = api.RenderData(scene, 192, 108, 1)
    assert rd_d.rd.instcnt == 4096
    gd = api.GpuRenderer(rd_d, max_depth=6, seed=2).upload()
    rng = np.random.default_rng(5)
    globs = scene.globs()
    moved = _move(globs, rng, 0.2, 1.0)
    globs[:] = moved
    rd_h.update_host()
    gh = api.GpuRenderer(rd_h, max_depth=6, seed=2).upload()
    gd.update_instances(moved)
    rays = np.concatenate([ol.random_rays(rd_d, 50000, seed=3, spread=20.0),
                           ol.camera_rays(rd_d)[::2]])
    info = _compare(gd, gh, rd_d, rd_h, rays, "stress build")
    print(f"stress device TLAS: {info[0]} nodes, depth {info[1]}")
    assert np.array_equal(_bits(_frame(gd, rd_d)), _bits(_frame(gh, rd_h)))
    gd.close()
    gh.close()
