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


def _host_tlas_sound(gr):
    """Upload the host-built TLAS; False when the upload rejects it.  The
    reference's build_bvh8 leaves an item count where a node offset belongs
    when a vertical split's partition comes out one-sided (rend.c:615-619),
    and the upload refuses such a tree."""
    try:
        gr.upload_dynamic()
        return True
    except api.RendgpuError as e:
        assert e.code == -1 and "offset" in str(e)
        return False


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
    gh = api.GpuRenderer(rd_h, max_depth=4, seed=5, ref_tlas=True).upload()
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
    # the one-CTA build collapsed by cost: another TLAS, the same hits; the
    # refit below then keeps its topology
    gd.update_instances(moved, tight=True, collapse=True)
    _, _, info_c = gd.instances()
    print(f"collapsed device TLAS: {info_c[0]} nodes, depth {info_c[1]}")
    assert info_c[2] == 0
    assert np.array_equal(_bits(gd.trace(rays)), _bits(gh.trace(rays)))
    assert np.array_equal(gd.occluded(rays), gh.occluded(rays))
    assert np.array_equal(_bits(_frame(gd, rd_d)), _bits(_frame(gh, rd_h)))
    # a small further move, refitted on the device (device matrices)
    import torch
    for s in range(10):
        moved2 = _move(moved, np.random.default_rng(100 + s), 0.02, 0.05)
        globs[:] = moved2
        rd_h.update_host()
        if _host_tlas_sound(gh):
            break
    else:
        pytest.fail("no move with a sound host TLAS")
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
    # rendgpu_upload_dynamic makes the uploaded instances current again
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
    gh = api.GpuRenderer(rd_h, max_depth=6, seed=2, ref_tlas=True).upload()
    gd.update_instances(moved)
    rays = np.concatenate([ol.random_rays(rd_d, 50000, seed=3, spread=20.0),
                           ol.camera_rays(rd_d)[::2]])
    info = _compare(gd, gh, rd_d, rd_h, rays, "stress build")
    print(f"stress device TLAS: {info[0]} nodes, depth {info[1]}")
    assert np.array_equal(_bits(_frame(gd, rd_d)), _bits(_frame(gh, rd_h)))
    gd.close()
    gh.close()


def test_device_build_where_the_host_build_fails(gpu):
    """A move after which the reference's TLAS build (restated byte for byte
    by the host library) writes a malformed tree: a vertical split whose
    partition comes out one-sided leaves the item count in place of a node
    offset (rend.c:615-619).  The upload rejects that tree; the device build
    handles the same matrices, and its closest hits hold the FP64
    brute-force closest hit over every instance whose box the ray enters."""
    scene = api.Scene(api.SCENE_SCALE, 3, 8)
    rd_d = api.RenderData(scene, 160, 90, 1)
    rd_h = api.RenderData(scene, 160, 90, 1)
    gd = api.GpuRenderer(rd_d, max_depth=4, seed=5).upload()
    gh = api.GpuRenderer(rd_h, max_depth=4, seed=5, ref_tlas=True).upload()
    rng = np.random.default_rng(11)
    globs = scene.globs()
    moved = _move(globs, rng, 0.3, 0.5)
    moved = _move(moved, rng, 0.02, 0.05)  # the host build fails here
    globs[:] = moved
    rd_h.update_host()
    assert not _host_tlas_sound(gh)
    with pytest.raises(api.RendgpuError):
        gh.trace(ol.random_rays(rd_h, 8))  # no half-uploaded scene
    gd.update_instances(moved)
    xf, wb, info = gd.instances()
    assert np.array_equal(_bits(xf), _bits(rd_h.globinv()))
    assert np.array_equal(_bits(wb), _bits(rd_h.aabbs()))
    assert info[2] == 0
    rays = np.concatenate([ol.random_rays(rd_d, 1500, seed=8),
                           ol.camera_rays(rd_d)[::20]])
    hits = gd.trace(rays)
    ok = ol.agrees_with_truth(rd_h.ptr, rays, hits)
    assert ok.mean() > 0.999, (ok.mean(), np.nonzero(~ok)[0][:5])
    assert (hits["t"] < ol.FLT_MAX).mean() > 0.1
    gd.close()
    gh.close()


@pytest.mark.parametrize("fam,param", [(api.SCENE_SCALE, 0),
                                       (api.SCENE_STRESS, 0)])
def test_upload_rebuild_matches_reference_tlas(gpu, fam, param):
    """By default rendgpu_upload_dynamic rebuilds the uploaded TLAS on the
    device over tight instance boxes; closest hits, any hits and frames are
    bit-identical to those through the converted reference TLAS
    (cfg.reserved[4] bit 0), and the tree is no deeper than the reference's
    (the traversal stack the upload sized still holds)."""
    scene = api.Scene(fam, 1, param)
    rd_t = api.RenderData(scene, 240, 135, 1)
    rd_r = api.RenderData(scene, 240, 135, 1)
    gt = api.GpuRenderer(rd_t, max_depth=6, seed=3).upload()
    gr = api.GpuRenderer(rd_r, max_depth=6, seed=3, ref_tlas=True).upload()
    # the same traversal stack (the rebuilt tree may use the levels that
    # stack has to spare beside the deepest BLAS)
    assert gt.get_tune()["stack"] == gr.get_tune()["stack"]
    rays = np.concatenate([ol.random_rays(rd_t, 60000, seed=6, spread=20.0),
                           ol.camera_rays(rd_t)[::2]])
    assert np.array_equal(_bits(gt.trace(rays)), _bits(gr.trace(rays)))
    assert np.array_equal(gt.occluded(rays), gr.occluded(rays))
    assert np.array_equal(_bits(_frame(gt, rd_t)), _bits(_frame(gr, rd_r)))
    gt.close()
    gr.close()
