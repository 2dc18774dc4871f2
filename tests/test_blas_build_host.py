"""The library's own BLAS build on the CPU (rendgpu_blas_host: the tree
rendgpu_upload_static builds, in host memory, without a GPU): every triangle
of the mesh in exactly one leaf with its vertices unchanged, child and item
indices in range, every quantised child box at least 1/32 of a quantum
outside the triangles below it, and the depth the build reports."""

import ctypes as C

import numpy as np
import pytest

from nodebleed_b200 import api

# struct nb_qnode / nb_gtri (gpulayout.h), struct rinst / rtri (rend.h)
QNODE = np.dtype([("p", "<f4", (3,)), ("e", "u1", (3,)), ("imask", "u1"),
                  ("child_base", "<u4"), ("item_base", "<u4"),
                  ("meta", "u1", (8,)), ("qlo", "u1", (3, 8)),
                  ("qhi", "u1", (3, 8))])
GTRI = np.dtype([("v0", "<f4", (3,)), ("prim", "<u4"), ("v1", "<f4", (3,)),
                 ("pad1", "<u4"), ("v2", "<f4", (3,)), ("pad2", "<u4")])
RINST = np.dtype([("globinv", "<f4", (12,)), ("flags", "<u4"),
                  ("triofs", "<u4"), ("tricnt", "<u4"), ("pad", "<u4")])
RTRI = np.dtype([("v0", "<f4", (3,)), ("p0", "<f4"), ("v1", "<f4", (3,)),
                 ("p1", "<f4"), ("v2", "<f4", (3,)), ("p2", "<f4")])
EXP_BIAS = 119  # stored exponent byte = e + 127 - 8 (qnode.h kQExpBias)
FRAME_MAX = 2.0 ** 125  # node frames are clamped here (qnode.h kQFrameMax)


def _array(ptr, dtype, n):
    raw = (C.c_ubyte * (dtype.itemsize * n)).from_address(ptr)
    return np.frombuffer(raw, dtype).copy()


def _build(rd, triofs, tricnt):
    g = api.gpu_lib().L
    info = (C.c_uint32 * 3)()
    assert g.rendgpu_blas_host(rd.ptr, triofs, tricnt, None, 0, None, 0,
                               info) == 0
    nodes = np.zeros(info[0], QNODE)
    tris = np.zeros(info[1], GTRI)
    assert g.rendgpu_blas_host(rd.ptr, triofs, tricnt, nodes.ctypes.data,
                               len(nodes), tris.ctypes.data, len(tris),
                               info) == 0
    return nodes, tris, int(info[2])


def _check(nodes, tris, depth, mesh):
    verts = np.stack([tris["v0"], tris["v1"], tris["v2"]], 1).astype(
        np.float64)                                   # (items, 3, 3)
    seen = np.zeros(len(mesh), np.int64)
    maxd = [0]

    def walk(ni, d):
        """Checks node ni; returns the bounds of its triangles."""
        assert 0 <= ni < len(nodes)
        maxd[0] = max(maxd[0], d)
        n = nodes[ni]
        scale = np.ldexp(1.0, n["e"].astype(np.int64) - EXP_BIAS)
        p = n["p"].astype(np.float64)
        lo_all = np.full(3, np.inf)
        hi_all = np.full(3, -np.inf)
        for s in range(8):
            inner = (int(n["imask"]) >> s) & 1
            meta = int(n["meta"][s])
            if inner:
                below = bin(int(n["imask"]) & ((1 << s) - 1)).count("1")
                clo, chi = walk(int(n["child_base"]) + below, d + 1)
            elif meta & 0x80:
                cnt = ((meta >> 5) & 3) + 1
                first = int(n["item_base"]) + (meta & 31)
                assert first + cnt <= len(tris)
                for k in range(first, first + cnt):
                    prim = int(tris["prim"][k])
                    seen[prim] += 1
                    t = mesh[prim]
                    for a, b in (("v0", "v0"), ("v1", "v1"), ("v2", "v2")):
                        assert np.array_equal(tris[a][k].view(np.uint32),
                                              t[b].view(np.uint32))
                v = verts[first:first + cnt].reshape(-1, 3)
                clo, chi = v.min(0), v.max(0)
            else:
                continue
            qlo = p + n["qlo"][:, s] * scale
            qhi = p + n["qhi"][:, s] * scale
            # contained unless the child reaches beyond the clamped frame
            inside = (clo >= -FRAME_MAX) & (chi <= FRAME_MAX)
            assert np.all((qlo <= clo - scale / 32) | ~inside), \
                (ni, s, qlo - clo)
            assert np.all((qhi >= chi + scale / 32) | ~inside), \
                (ni, s, qhi - chi)
            assert np.all(np.isfinite(qlo) & np.isfinite(qhi))
            lo_all = np.minimum(lo_all, clo)
            hi_all = np.maximum(hi_all, chi)
        assert np.isfinite(lo_all).all(), f"node {ni} without children"
        return lo_all, hi_all

    walk(0, 1)
    assert np.all(seen == 1), np.nonzero(seen != 1)[0][:5]
    assert maxd[0] == depth


@pytest.mark.parametrize("fam,param", [(api.SCENE_TINY, 0),
                                       (api.SCENE_SCALE, 3)])
def test_blas_build_host(fam, param):
    scene = api.Scene(fam, 1, param)
    rd = api.RenderData(scene, 64, 36, 1)
    insts = _array(rd.rd.insts, RINST, rd.rd.instcnt)
    meshes = sorted({(int(i["triofs"]), int(i["tricnt"])) for i in insts})
    total = sum(c for _, c in meshes)
    alltris = _array(rd.rd.tris, RTRI, max(o + c for o, c in meshes))
    for triofs, tricnt in meshes:
        nodes, tris, depth = _build(rd, triofs, tricnt)
        assert len(tris) == tricnt and depth >= 1
        _check(nodes, tris, depth, alltris[triofs:triofs + tricnt])
    assert total > 0
    rd.close()
    scene.close()


def test_blas_build_host_rejects_bad_arguments():
    g = api.gpu_lib().L
    info = (C.c_uint32 * 3)()
    assert g.rendgpu_blas_host(None, 0, 1, None, 0, None, 0, info) == -1
    scene = api.Scene(api.SCENE_TINY, 1)
    rd = api.RenderData(scene, 16, 9, 1)
    assert g.rendgpu_blas_host(rd.ptr, 0, 0, None, 0, None, 0, info) == -1
    rd.close()
    scene.close()


def _writable(ptr, dtype, n):
    raw = (C.c_ubyte * (dtype.itemsize * n)).from_address(ptr)
    return np.frombuffer(raw, dtype)


def _planted(kind, n, rng):
    """n triangles (n, 3 vertices, xyz) of one degenerate or extreme kind."""
    if kind == "identical":      # every centroid and box the same
        return np.broadcast_to(rng.normal(size=(1, 3, 3)), (n, 3, 3))
    if kind == "points":         # zero-size boxes on a line, duplicates
        p = np.zeros((n, 1, 3))
        p[:, 0, 0] = rng.integers(0, 7, n)
        return np.broadcast_to(p, (n, 3, 3))
    if kind == "flat":           # zero extent along z
        v = rng.normal(size=(n, 3, 3))
        v[:, :, 2] = 0.5
        return v
    if kind == "huge":
        return rng.normal(size=(n, 3, 3)) * 1e30
    if kind == "tiny":
        return rng.normal(size=(n, 3, 3)) * 1e-30
    if kind == "fltmax":         # next to the float range's ends
        return rng.uniform(-1.0, 1.0, (n, 3, 3)) * 3.4e38
    if kind == "beyond":         # half wholly outside the 2^125 frame
        v = rng.uniform(0.0, 1.0, (n, 3, 3))
        v[: (n + 1) // 2] = 1e38 + v[: (n + 1) // 2] * 2.4e38
        return v
    if kind == "mixed":          # small triangles inside huge node boxes
        v = rng.normal(size=(n, 3, 3))
        v[: n // 2] *= 1e20
        v[n // 2:] = v[n // 2:] * 1e-3 + 1.0
        return v
    return rng.normal(size=(n, 3, 3)) * rng.uniform(0.01, 10.0, (n, 1, 1))


@pytest.mark.timeout(120)
@pytest.mark.parametrize("kind", ["identical", "points", "flat", "huge",
                                  "tiny", "mixed", "fltmax", "beyond",
                                  "random"])
@pytest.mark.parametrize("count", [1, 2, 5, 9, 128, 129, 320])
def test_blas_build_host_degenerate_and_extreme(kind, count):
    """Planted meshes: one instance's range cut to `count` triangles (the
    sweep / binned split boundary at 128 included) and its triangles
    replaced by coincident, point-like, flat, huge, tiny, mixed-scale or
    near-FLT_MAX ones; the tree must still hold every triangle once inside
    conservative boxes (the build must end: an unbounded exponent search
    once spun on infinite frames)."""
    scene = api.Scene(api.SCENE_TINY, 1)
    rd = api.RenderData(scene, 16, 9, 1)
    insts = _writable(rd.rd.insts, RINST, rd.rd.instcnt)
    big = int(np.argmax(insts["tricnt"]))
    triofs = int(insts["triofs"][big])
    assert count <= int(insts["tricnt"][big])
    insts["tricnt"][big] = count
    rng = np.random.default_rng(count * 31 + len(kind))
    v = _planted(kind, count, rng).astype(np.float32)
    tris = _writable(rd.rd.tris, RTRI, triofs + count)[triofs:]
    for k, name in enumerate(("v0", "v1", "v2")):
        tris[name] = v[:, k]
    mesh = tris.copy()
    nodes, out, depth = _build(rd, triofs, count)
    assert len(out) == count and depth >= 1
    _check(nodes, out, depth, mesh)
    rd.close()
    scene.close()


def test_blas_build_host_rejects_unknown_ranges_and_nan():
    scene = api.Scene(api.SCENE_TINY, 1)
    rd = api.RenderData(scene, 16, 9, 1)
    g = api.gpu_lib().L
    info = (C.c_uint32 * 3)()
    insts = _writable(rd.rd.insts, RINST, rd.rd.instcnt)
    triofs, tricnt = int(insts["triofs"][0]), int(insts["tricnt"][0])
    # a range no instance uses (it could run past the triangle array)
    assert g.rendgpu_blas_host(rd.ptr, triofs, tricnt + 1, None, 0, None, 0,
                               info) == -1
    assert g.rendgpu_blas_host(rd.ptr, triofs + 1, tricnt, None, 0, None, 0,
                               info) == -1
    tris = _writable(rd.rd.tris, RTRI, triofs + tricnt)
    tris["v1"][triofs + tricnt - 1] = np.float32("nan")
    assert g.rendgpu_blas_host(rd.ptr, triofs, tricnt, None, 0, None, 0,
                               info) == -1
    rd.close()
    scene.close()
