"""GPU wavefront frames (rendgpu_render) against the CPU oracle's path
tracer on the same PCG32 streams."""

import numpy as np
import pytest

from nodebleed_b200 import api
import oracle_lib as ol

pytestmark = pytest.mark.gpu


def relmse(x, ref):
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2)))


def _gpu_frame(rd, depth, mode, seed):
    """One GPU frame; rd.samples is left at its value before the frame so
    the oracle renders the same random streams."""
    gr = api.GpuRenderer(rd, max_depth=depth, mode=mode, seed=seed).upload()
    samples = rd.rd.samples
    rays = gr.frame()
    rd.rd.samples = samples
    gr.readback(3)
    acc = rd.acc().copy()
    lights, area = gr.lights()
    gr.close()
    return acc, rays, lights, area


@pytest.mark.parametrize("fam,seed,depth", [
    (api.SCENE_TINY, 1, 3), (api.SCENE_TINY, 2, 5), (api.SCENE_SMALL, 1, 2),
    (api.SCENE_GLOSSY, 1, 6), (api.SCENE_GLOSSY, 2, 8)])
def test_path_frame_matches_oracle(gpu, fam, seed, depth):
    scene = api.Scene(fam, seed)
    rd = api.RenderData(scene)
    if fam == api.SCENE_SMALL:
        rd.resize(160, 90, 1)
    acc, rays, lights, area = _gpu_frame(rd, depth, api.MODE_PATH, 11)
    rad, orays = ol.orc_render(rd, lights, area, depth, seed=11)
    same = np.all(acc == rad, axis=2).mean()
    assert same > 0.98, same
    assert relmse(acc, rad) < 2e-3
    assert abs(int(rays) - int(orays)) <= 0.01 * orays


def test_primary_frame_matches_oracle(gpu):
    scene = api.Scene(api.SCENE_SMALL, 1)
    rd = api.RenderData(scene)
    rd.resize(320, 180, 2)
    acc, rays, _, _ = _gpu_frame(rd, 1, api.MODE_PRIMARY, 5)
    rad, orays = ol.orc_render(rd, np.zeros((0, 20), np.float32), 0.0, 1,
                               mode=1, seed=5)
    assert rays == orays == 320 * 180 * 2
    assert np.all(acc == rad, axis=2).mean() > 0.995


def test_accumulation_and_argb8(gpu):
    scene = api.Scene(api.SCENE_TINY, 3)
    rd = api.RenderData(scene)
    gr = api.GpuRenderer(rd, max_depth=3, seed=2).upload()
    lights, area = gr.lights()
    # two frames on the GPU, two oracle frames accumulated the same way
    ref = api.RenderData(api.Scene(api.SCENE_TINY, 3))
    for _ in range(2):
        rad, _ = ol.orc_render(ref, lights, area, 3, seed=2)
        ol.oracle().orc_accumulate(ref.ptr, rad.ctypes.data)
        ref.rd.samples += ref.rd.spp
        gr.frame()
    gr.readback(3)
    same = np.all(rd.acc() == ref.acc(), axis=2)
    assert same.mean() > 0.98
    assert (rd.buf[same.ravel()] == ref.buf[same.ravel()]).all()
    assert rd.rd.samples == 2
    gr.close()


def test_light_table_matches_independent_fp64(gpu):
    from test_oracle import _lights_numpy
    scene = api.Scene(api.SCENE_SCALE, 1, 4)
    rd = api.RenderData(scene)
    gr = api.GpuRenderer(rd).upload()
    lights, area = gr.lights()
    ref, ref_area = _lights_numpy(rd)
    assert lights.shape == ref.shape
    assert np.allclose(lights, ref, rtol=1e-5, atol=1e-5)
    assert abs(area - ref_area) < 1e-4 * ref_area
    gr.close()


def test_frame_claim_and_ray_count(gpu):
    """rendgpu_render has the thrd_start_t shape: the first caller of a
    frame renders, later callers of the same frame return at once."""
    scene = api.Scene(api.SCENE_TINY, 1)
    rd = api.RenderData(scene)
    gr = api.GpuRenderer(rd, max_depth=2).upload()
    g = gr.g
    g.rendgpu_render(rd.ptr)
    rays1 = rd.rd.rays
    assert rays1 > 0 and rd.rd.blknum == 1
    g.rendgpu_render(rd.ptr)  # same frame: no second render
    assert rd.rd.rays == rays1 and rd.rd.blknum == 2
    gr.close()


def _tonemap_fp64(acc, samples, op, exposure):
    """The tonemapped 8-bit resolve restated in FP64 after the FP32
    exposure product: Reinhard (op 1) or Narkowicz's ACES fit (op 2), the
    sRGB transfer function, round to nearest, clamp to 0..255."""
    inv = np.float32(1.0) / np.float32(samples)
    e = np.float32(inv * np.float32(exposure))
    v = np.maximum((acc.astype(np.float32) * e).astype(np.float64), 0.0)
    if op == 1:
        v = v / (1.0 + v)
    else:
        v = np.minimum(v * (2.51 * v + 0.03) / (v * (2.43 * v + 0.59) + 0.14),
                       1.0)
    s = np.where(v <= 0.0031308, 12.92 * v, 1.055 * v ** (1 / 2.4) - 0.055)
    return np.clip(np.rint(s * 255.0), 0, 255).astype(np.int64)


@pytest.mark.parametrize("op", [api.RESOLVE_REINHARD, api.RESOLVE_ACES])
def test_tonemapped_resolve(gpu, op):
    scene = api.Scene(api.SCENE_TINY, 3)
    rd = api.RenderData(scene)
    gr = api.GpuRenderer(rd, max_depth=3, seed=2).upload()
    gr.set_resolve(op, 1.5)
    for _ in range(2):
        gr.frame()
    gr.readback(3)
    acc, buf = rd.acc(), rd.buf.reshape(rd.rd.height, rd.rd.width)
    want = _tonemap_fp64(acc, rd.rd.samples, op, 1.5)
    got = np.stack([(buf >> 16) & 255, (buf >> 8) & 255, buf & 255],
                   axis=2).astype(np.int64)
    assert ((buf >> 24) == 255).all()
    diff = np.abs(got - want)
    # powf on the device against FP64 pow: at most one 8-bit step apart
    assert diff.max() <= 1, diff.max()
    assert (diff == 0).mean() > 0.99
    assert want.max() > 128  # the image is not black
    # back to the reference's wrapping pack (rend.c:3574-3577)
    gr.set_resolve(api.RESOLVE_WRAP)
    gr.frame()
    gr.readback(3)
    acc, buf = rd.acc(), rd.buf.reshape(rd.rd.height, rd.rd.width)
    inv = np.float32(1.0) / np.float32(rd.rd.samples)
    wrap = ((np.float32(255.0) * (acc * inv)).astype(np.uint32) & 255)
    got = np.stack([(buf >> 16) & 255, (buf >> 8) & 255, buf & 255], axis=2)
    assert np.array_equal(got, wrap)
    with pytest.raises(api.RendgpuError):
        gr.set_resolve(3)
    gr.close()


def test_gltf_scene_renders_like_the_in_memory_scene(gpu, tmp_path):
    """Config 1 written as .gltf + .bin and loaded back by the host library
    (nbh_scene_load_gltf) renders the same frame, bit for bit, as the scene
    it was written from (640x360, 1 spp, depth 5)."""
    src = api.Scene(api.SCENE_SMALL, 1)
    path = str(tmp_path / "config1.gltf")
    src.save_gltf(path)
    got = api.Scene.load_gltf(path)
    accs = []
    for sc in (src, got):
        rd = api.RenderData(sc, 640, 360, 1)
        acc, rays, _, _ = _gpu_frame(rd, 5, api.MODE_PATH, 9)
        assert rays > 640 * 360
        accs.append(acc)
        rd.close()
    assert np.array_equal(accs[0].view(np.uint32), accs[1].view(np.uint32))
