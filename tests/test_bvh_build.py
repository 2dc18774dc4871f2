"""The host BVH8 build restatement produces the reference's node bytes
(rend.c:458-709, 3033-3090)."""

import ctypes as C
import os

import numpy as np
import pytest

from nodebleed_b200 import api
import oracle_lib as ol
from golden.make_golden import bvh_digest, ref_rdata, scene_digest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("name", ["tiny_s1", "small_s1", "scale_s1_b4"])
def test_build_matches_golden_digest(name):
    g = np.load(os.path.join(HERE, "golden", name + ".npz"))
    scene = api.Scene(int(g["family"]), int(g["seed"]), int(g["param"]))
    rd = api.RenderData(scene)
    assert scene_digest(rd) == str(g["scene_sha"])
    assert bvh_digest(rd) == str(g["bvh_sha"])


@pytest.mark.parametrize("family,seed,param", [
    (api.SCENE_TINY, 2, 0), (api.SCENE_TINY, 3, 6),
    (api.SCENE_SMALL, 2, 16), (api.SCENE_BATCH, 1, 3),
    (api.SCENE_SCALE, 2, 3)])
def test_build_matches_reference_build(family, seed, param):
    if ol.ref() is None:
        pytest.skip("reference build not present")
    scene = api.Scene(family, seed, param)
    if scene.tris > 400000:
        pytest.skip("large scene")
    mine = api.RenderData(scene)
    theirs = ref_rdata(scene)
    assert bvh_digest(mine) == bvh_digest(theirs)


def test_build_invariants_small():
    """Every triangle lands in exactly one leaf; child boxes bound their
    triangles; empty child slots have inverted boxes."""
    scene = api.Scene(api.SCENE_SMALL, 1, 8)
    rd = api.RenderData(scene)
    r = rd.rd
    n = 2 * (scene.tris + r.instcnt)
    raw = np.ctypeslib.as_array((C.c_ubyte * (n * 256)).from_address(
        r.bnodes))
    tris = np.ctypeslib.as_array((C.c_float * (scene.tris * 12)).from_address(
        r.tris)).reshape(-1, 12)
    # first BLAS: triofs 0, tricnt from instance 0
    insts = np.ctypeslib.as_array((C.c_uint32 * (16 * r.instcnt)).from_address(
        r.insts)).reshape(-1, 16)
    triofs, tricnt = insts[0, 13], insts[0, 14]
    base = 2 * triofs * 256
    seen = np.zeros(tricnt, np.int32)
    stack = [0]
    while stack:
        ofs = stack.pop()
        node = raw[base + ofs: base + ofs + 256]
        f = node[:192].view(np.float32).reshape(6, 8)
        ch = node[192:224].view(np.uint32)
        for j in range(8):
            mn = f[[0, 2, 4], j]
            mx = f[[1, 3, 5], j]
            if (mn > mx).any():
                continue
            if ch[j] & 0x80000000:
                lo = base + (int(ch[j]) & 0x7fffffff)
                leaf = raw[lo:lo + 192]
                ids = leaf[144:160].view(np.uint32)
                cnt = int(leaf[160:164].view(np.uint32)[0])
                assert 1 <= cnt <= 4
                for k in range(cnt):
                    seen[ids[k]] += 1
                    v = tris[triofs + ids[k]].reshape(3, 4)[:, :3]
                    assert (v.min(0) >= mn - 1e-6).all()
                    assert (v.max(0) <= mx + 1e-6).all()
            else:
                stack.append(int(ch[j]))
    assert (seen == 1).all()


def test_scene_generator_rejects_unknown_family_and_oversized_params():
    """nbh_scene_gen returns -1 (RuntimeError here) for an unknown family
    and for params above NBH_MAX_SPHERE_FREQ (SMALL/TINY) or NBH_MAX_BLAS
    (SCALE/STRESS/GLOSSY), instead of generating an unbounded scene."""
    for fam, param in ((7, 0), (api.SCENE_TINY, 1025),
                       (api.SCENE_SMALL, 1 << 31),
                       (api.SCENE_SCALE, 4097),
                       (api.SCENE_STRESS, 0xffffffff)):
        with pytest.raises(RuntimeError):
            api.Scene(fam, 1, param)
    # params within the bounds still generate
    s = api.Scene(api.SCENE_TINY, 1, 8)
    assert s.tris > 0
    s.close()
