"""Generate the golden fixtures of the parity tests from the reference.

Runs the reference renderer compiled from its own sources
(oracle/_ref/libnbref.so, built by `make -C oracle ref` where the reference
sources are present) on seeded synthetic scenes and stores, per scene:

* sha256 of the scene's triangles and of the BVH bytes the reference's
  rend_prepstatic/rend_prepdynamic produce (rend.c:3033/3073);
* a ray set: the reference's own camera rays (make_camray_pckt, rend.c:3293)
  plus random rays, and the reference hits of intersect_tlas (rend.c:1976)
  and intersect_pckts_tlas (rend.c:2472) on them;
* occlusion answers of intersect_any_tlas (rend.c:2883) on rays with a
  finite tmax;
* for the tiny scene, one frame of the live renderer rend_render
  (rend.c:3603): the accumulator and the ARGB8 image.

Usage: python tests/golden/make_golden.py   (writes tests/golden/*.npz)
"""

import ctypes as C
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from nodebleed_b200 import api  # noqa: E402
import oracle_lib as ol  # noqa: E402


def scene_digest(rd):
    r = rd.rd
    ntri = rd.scene.tris
    tris = (C.c_ubyte * (48 * ntri)).from_address(r.tris)
    return hashlib.sha256(bytes(tris)).hexdigest()


def bvh_digest(rd):
    r = rd.rd
    n = 2 * (rd.scene.tris + r.instcnt) * 256
    nodes = (C.c_ubyte * n).from_address(r.bnodes)
    return hashlib.sha256(bytes(nodes)).hexdigest()


def ref_rdata(scene):
    """Render data whose BVHs come from the reference's own build."""
    R = ol.ref()
    h = api.host_lib().L
    rd = api.RenderData.__new__(api.RenderData)
    rd.h = h
    rd.scene = scene
    rd.ptr = h.nbh_rdata_new()
    s = scene.s
    h.nbh_rend_init(rd.ptr, max(s.mtlcnt, 1), scene.tris, s.instcnt, s.spp)
    h.nbh_cpy_rdata(rd.ptr, scene.ptr)
    R.rend_prepstatic(rd.ptr)
    h.nbh_upd_rinsts(rd.ptr, scene.ptr)
    R.rend_prepdynamic(rd.ptr)
    h.nbh_rend_resaccum(rd.ptr, s.width, s.height)
    camp = C.addressof(scene.s) + api.SceneStruct.cam.offset
    h.nbh_upd_rcam(rd.ptr, camp, float(s.width), float(s.height))
    rd.attach_buf()
    return rd


def ref_camera_rays(rd, npckts, seed):
    """Camera rays of the reference (make_camray_pckt), packets at random
    4x2-aligned pixel positions."""
    R = ol.ref()
    r = rd.rd
    rng = np.random.default_rng(seed)
    px = (rng.integers(0, r.width // 4, npckts) * 4).astype(np.uint32)
    py = (rng.integers(0, r.height // 2, npckts) * 2).astype(np.uint32)
    pxy = np.ascontiguousarray(np.stack([px, py], 1).ravel(), np.uint32)
    out = np.zeros(npckts * 8, api.RAY_DTYPE)
    R.refh_camrays(rd.ptr, 0, 0, (seed + 13) * 1571, 23, npckts,
                   pxy.ctypes.data, out.ctypes.data)
    return out


def make(name, family, seed, param, n_random, n_pckts, frame=False):
    scene = api.Scene(family, seed, param)
    rd = ref_rdata(scene)
    cam = ref_camera_rays(rd, n_pckts, seed)
    rnd = ol.random_rays(rd, n_random, seed=seed)
    rays = np.concatenate([cam, rnd])
    hits = ol.ref_trace(rd.ptr, rays)
    pk = ol.ref_trace(rd.ptr, cam, packets=True)
    # shadow-like rays: random rays with tmax at a random fraction of the
    # reference hit distance (or 10 for misses)
    rng = np.random.default_rng(seed + 7)
    sh = rnd.copy()
    th = hits["t"][len(cam):]
    sh["tmax"] = np.where(th < ol.FLT_MAX, th * rng.uniform(0.5, 1.5, len(sh)),
                          10.0).astype(np.float32)
    occl = ol.ref_occluded(rd.ptr, sh)
    out = dict(scene_sha=scene_digest(rd), bvh_sha=bvh_digest(rd),
               family=family, seed=seed, param=param, rays=rays, hits=hits,
               pckt_rays=cam, pckt_hits=pk, shadow_rays=sh, occl=occl)
    if frame:
        R = ol.ref()
        rays_n = R.refh_render_frame(rd.ptr, 4)
        out["frame_acc"] = rd.acc().copy()
        out["frame_buf"] = rd.buf.copy()
        out["frame_rays"] = rays_n
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, len(rays), "rays,", int((hits["t"] < ol.FLT_MAX).sum()),
          "hits", out["bvh_sha"][:12])
    rd.close()
    scene.close()


if __name__ == "__main__":
    if ol.ref() is None:
        sys.exit("oracle/_ref/libnbref.so missing: run make -C oracle ref")
    make("tiny_s1", api.SCENE_TINY, 1, 0, 4096, 256, frame=True)
    make("small_s1", api.SCENE_SMALL, 1, 0, 8192, 512)
    make("scale_s1_b4", api.SCENE_SCALE, 1, 4, 8192, 512)
