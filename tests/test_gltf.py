"""glTF 2.0 scenes through the host library (nbh_scene_load_gltf /
nbh_scene_save_gltf), CPU only.

* Round trip: the config-1 scene written as .gltf + .bin and loaded back
  gives render data byte-identical to the in-memory scene's, and the
  oracle renders the same image from both.
* The loader against nodebleed's own importer (imp_gltf_f, gltfimp.c:415,
  compiled into oracle/_ref) on the same file, read without this library's
  exact-transform extras: vertices, normals, indices, per-triangle
  materials and materials bit-identical; node world matrices and the
  camera within FP32 rounding of the two ways of composing them.
"""

import ctypes as C
import os

import numpy as np
import pytest

from nodebleed_b200 import api
import oracle_lib as ol


class MeshStruct(C.Structure):
    """struct nbh_mesh (nb_host.h)."""
    _fields_ = [("vcnt", C.c_uint32), ("vrts", C.c_void_p),
                ("nrms", C.c_void_p), ("icnt", C.c_uint32),
                ("inds", C.c_void_p), ("mtlid", C.c_uint32),
                ("tmtl", C.c_void_p)]


def _arr(ptr, n, dtype):
    if n == 0:
        return np.zeros(0, dtype)
    raw = (C.c_ubyte * (n * np.dtype(dtype).itemsize)).from_address(ptr)
    return np.frombuffer(bytes(raw), dtype)


def _meshes(sc):
    ms = (MeshStruct * sc.s.meshcnt).from_address(sc.s.meshes)
    out = []
    for m in ms:
        tm = (_arr(m.tmtl, m.icnt // 3, np.uint32) if m.tmtl else
              np.full(m.icnt // 3, m.mtlid, np.uint32))
        out.append((_arr(m.vrts, 3 * m.vcnt, np.float32),
                    _arr(m.nrms, 3 * m.vcnt, np.float32),
                    _arr(m.inds, m.icnt, np.uint32), tm))
    return out


def _rdata_bytes(rd, scene):
    r = rd.rd
    nt = scene.tris
    return {"tris": _arr(r.tris, 12 * nt, np.uint32),
            "nrms": _arr(r.nrms, 12 * nt, np.uint32),
            "mtls": _arr(r.mtls, 8 * scene.s.mtlcnt, np.uint32),
            "insts": _arr(r.insts, 16 * r.instcnt, np.uint32),
            "aabbs": _arr(r.aabbs, 8 * r.instcnt, np.uint32),
            "cam": np.frombuffer(bytes(r.cam), np.uint32),
            "bg": np.frombuffer(bytes(r.bgcol), np.uint32)}


def test_round_trip_is_exact(tmp_path):
    from test_oracle import _lights_numpy
    src = api.Scene(api.SCENE_SMALL, 1)
    path = str(tmp_path / "small.gltf")
    src.save_gltf(path)
    assert os.path.exists(str(tmp_path / "small.bin"))
    got = api.Scene.load_gltf(path)
    assert (got.s.meshcnt, got.s.mtlcnt, got.s.instcnt) == \
        (src.s.meshcnt, src.s.mtlcnt, src.s.instcnt)
    w, h = 96, 54
    rd_a = api.RenderData(src, w, h, 1)
    rd_b = api.RenderData(got, w, h, 1)
    a, b = _rdata_bytes(rd_a, src), _rdata_bytes(rd_b, got)
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    # the oracle's path tracer renders the same image from both
    la, aa = _lights_numpy(rd_a)
    lb, ab = _lights_numpy(rd_b)
    img_a, _ = ol.orc_render(rd_a, la, aa, 5, seed=3)
    img_b, _ = ol.orc_render(rd_b, lb, ab, 5, seed=3)
    assert np.array_equal(img_a, img_b)
    assert img_a.max() > 0


def test_loader_matches_reference_importer(tmp_path):
    R = ol.ref()
    if R is None:
        pytest.skip("reference build not present")
    vp, u32 = C.c_void_p, C.c_uint32
    R.refh_gltf_import.argtypes = [C.c_char_p] + [vp] * 9
    src = api.Scene(api.SCENE_SMALL, 2)
    path = str(tmp_path / "small2.gltf")
    src.save_gltf(path)
    counts = (u32 * 5)()
    R.refh_gltf_import(os.fsencode(path), counts, *([None] * 8))
    nm, nv, ni, nmt, nn = list(counts)
    vrts = np.zeros(3 * nv, np.float32)
    nrms = np.zeros(3 * nv, np.float32)
    inds = np.zeros(ni, np.uint32)
    trimtl = np.zeros(ni // 3, np.uint32)
    mtls = np.zeros(7 * nmt, np.float32)
    node_mesh = np.zeros(nn, np.uint32)
    globs = np.zeros(16 * nn, np.float32)
    cam = np.zeros(13, np.float32)
    R.refh_gltf_import(os.fsencode(path), counts, vrts.ctypes.data,
                       nrms.ctypes.data, inds.ctypes.data,
                       trimtl.ctypes.data, mtls.ctypes.data,
                       node_mesh.ctypes.data, globs.ctypes.data,
                       cam.ctypes.data)
    ours = api.Scene.load_gltf(path, extras=False)
    om = _meshes(ours)
    assert len(om) == nm
    assert np.array_equal(np.concatenate([m[0] for m in om]).view(np.uint32),
                          vrts.view(np.uint32))
    assert np.array_equal(np.concatenate([m[1] for m in om]).view(np.uint32),
                          nrms.view(np.uint32))
    assert np.array_equal(np.concatenate([m[2] for m in om]), inds)
    assert np.array_equal(np.concatenate([m[3] for m in om]), trimtl)
    om_ = _arr(ours.s.mtls, 8 * nmt, np.float32).reshape(nmt, 8)
    ref_m = mtls.reshape(nmt, 7)
    assert np.array_equal(om_[:, :6].view(np.uint32),
                          ref_m[:, :6].view(np.uint32))
    emissive = 0x1000
    assert np.array_equal(om_[:, 6].view(np.uint32) & emissive,
                          ref_m[:, 6].view(np.uint32) & emissive)
    assert (om_[:, 6].view(np.uint32) & emissive).any()  # the quad light
    # instances: same meshes, world matrices within FP32 rounding
    assert ours.s.instcnt == nn
    ig = ours.globs()
    raw = (C.c_ubyte * (72 * nn)).from_address(ours.s.insts)
    imesh = np.frombuffer(bytes(raw), np.uint32).reshape(nn, 18)[:, 0]
    assert np.array_equal(imesh, node_mesh)
    assert np.allclose(ig, globs.reshape(nn, 16), rtol=1e-5, atol=1e-5)
    # and the generator's own matrices, which the TRS were written from
    assert np.allclose(ig, src.globs(), rtol=1e-5, atol=1e-5)
    oc = np.frombuffer(bytes(ours.s.cam), np.float32)
    ours_cam = np.concatenate([oc[0:3], oc[4:7], oc[8:11], oc[12:15],
                               oc[3:4]])
    assert np.allclose(ours_cam, cam, rtol=1e-5, atol=1e-5)


def test_reference_built_render_data(tmp_path):
    """The same file through nodebleed's own host code end to end
    (refh_gltf_rdata: imp_gltf_f, rend_init, the main.c copy, rend_prepstatic,
    upd_rinsts with its mat4_inv, rend_prepdynamic, upd_rcam) against this
    library's loader and bridge: triangles, normals, materials and every BLAS
    byte-identical; instance matrices, boxes and camera within the FP32
    rounding of the two matrix paths; the oracle's image of both alike."""
    if ol.ref() is None:
        pytest.skip("reference build not present")
    from test_oracle import _lights_numpy
    src = api.Scene(api.SCENE_SMALL, 1)
    path = str(tmp_path / "config1.gltf")
    src.save_gltf(path)
    w, h = 160, 90
    ref_rd = ol.RefRenderData(path, w, h, 1)
    ours = api.Scene.load_gltf(path, extras=False)
    rd = api.RenderData(ours, w, h, 1)
    r, q = ref_rd.rd, rd.rd
    assert (r.instcnt, r.width, r.height, r.spp) == \
        (q.instcnt, q.width, q.height, q.spp)
    nt = ours.tris
    # every word but the pads, which main.c leaves as rend_init's malloc
    # left them
    used = {"tris": [0, 1, 2, 4, 5, 6, 8, 9, 10],
            "nrms": [0, 1, 2, 3, 4, 5, 6, 8, 9, 10]}
    for f, cols in used.items():
        a = _arr(getattr(r, f), 12 * nt, np.uint32).reshape(nt, 12)
        b = _arr(getattr(q, f), 12 * nt, np.uint32).reshape(nt, 12)
        assert np.array_equal(a[:, cols], b[:, cols]), f
    nm = ours.s.mtlcnt
    # the pad word differs: main.c copies sizeof(struct rmtl) = 32 bytes
    # from each 28-byte struct mtl, so its pad holds the next material's
    # first word; nothing reads it
    assert np.array_equal(_arr(r.mtls, 8 * nm, np.uint32).reshape(nm, 8)[:, :7],
                          _arr(q.mtls, 8 * nm, np.uint32).reshape(nm, 8)[:, :7])
    ri = _arr(r.insts, 16 * r.instcnt, np.uint32).reshape(-1, 16)
    qi = _arr(q.insts, 16 * q.instcnt, np.uint32).reshape(-1, 16)
    assert np.array_equal(ri[:, 12:15], qi[:, 12:15])  # flags, triofs, cnt
    for ofs, cnt in {(int(a[13]), int(a[14])) for a in qi}:
        nb = 2 * cnt * 256
        assert np.array_equal(_arr(r.bnodes + 512 * ofs, nb, np.uint8),
                              _arr(q.bnodes + 512 * ofs, nb, np.uint8)), ofs
    assert np.allclose(ri[:, :12].view(np.float32),
                       qi[:, :12].view(np.float32), rtol=1e-4, atol=1e-5)
    assert np.allclose(_arr(r.aabbs, 8 * r.instcnt, np.float32),
                       _arr(q.aabbs, 8 * q.instcnt, np.float32),
                       rtol=1e-4, atol=1e-4)
    assert np.allclose(np.frombuffer(bytes(r.cam), np.float32)[:16],
                       np.frombuffer(bytes(q.cam), np.float32)[:16],
                       rtol=1e-5, atol=1e-5)
    assert np.array_equal(np.frombuffer(bytes(r.bgcol), np.uint32),
                          np.frombuffer(bytes(q.bgcol), np.uint32))
    lights, area = _lights_numpy(rd)
    img_r, _ = ol.orc_render(ref_rd, lights, area, 5, seed=4)
    img_q, _ = ol.orc_render(rd, lights, area, 5, seed=4)
    err = np.mean((img_r - img_q) ** 2 / (img_q ** 2 + 1e-2))
    assert err < 1e-4, err
    assert np.all(img_r == img_q, axis=2).mean() > 0.5
    ref_rd.close()
    rd.close()


def test_loader_rejects_malformed(tmp_path):
    bad = tmp_path / "bad.gltf"
    bad.write_text('{"asset": {"version": "2.0"}, "meshes": [')
    with pytest.raises(RuntimeError):
        api.Scene.load_gltf(str(bad))
    missing = tmp_path / "nobin.gltf"
    missing.write_text('{"buffers": [{"uri": "absent.bin"}], "meshes": []}')
    with pytest.raises(RuntimeError):
        api.Scene.load_gltf(str(missing))


def _corruptions(doc, binlen):
    """(name, edit of the parsed .gltf, expected: 'error' or 'loads')."""
    import copy
    nacc = len(doc["accessors"])
    idx_acc = doc["meshes"][0]["primitives"][0]["indices"]
    nnodes = len(doc["nodes"])

    def edit(f):
        def run(d):
            d = copy.deepcopy(d)
            f(d)
            return d
        return run

    def chain(d, shared):
        # nodes nnodes.. nnodes+39: each lists the next as its children
        # (twice when shared), reached from the scene root
        base = len(d["nodes"])
        for i in range(40):
            nxt = [base + i + 1] * (2 if shared else 1) if i < 39 else []
            d["nodes"].append({"children": nxt} if nxt else {})
        d["scenes"][d.get("scene", 0)]["nodes"].append(base)

    def cycle(d):
        d["nodes"][0].setdefault("children", []).append(0)

    def root_twice(d):
        roots = d["scenes"][d.get("scene", 0)]["nodes"]
        roots.append(roots[0])

    return [
        ("huge accessor count", edit(lambda d: d["accessors"][0].update(
            count=10 ** 9)), "error"),
        ("view past the buffer", edit(lambda d: d["bufferViews"][0].update(
            byteOffset=binlen)), "error"),
        ("view longer than the buffer", edit(
            lambda d: d["bufferViews"][-1].update(byteLength=binlen * 4)),
         "loads"),
        ("accessor offset past its view", edit(
            lambda d: d["accessors"][idx_acc].update(byteOffset=1 << 30)),
         "error"),
        ("index count not a multiple of 3", edit(
            lambda d: d["accessors"][idx_acc].update(
                count=d["accessors"][idx_acc]["count"] - 1)), "error"),
        ("float indices", edit(lambda d: d["accessors"][idx_acc].update(
            componentType=5126)), "error"),
        ("positions as VEC2", edit(lambda d: d["accessors"][
            d["meshes"][0]["primitives"][0]["attributes"]["POSITION"]
        ].update(type="VEC2")), "error"),
        ("accessor out of range", edit(
            lambda d: d["meshes"][0]["primitives"][0].update(
                indices=nacc + 5)), "error"),
        ("mesh out of range", edit(lambda d: [
            n.update(mesh=len(d["meshes"]) + 3) for n in d["nodes"]
            if "mesh" in n][:1]), "error"),
        ("material out of range (the first material instead)", edit(
            lambda d: d["meshes"][0]["primitives"][0].update(material=999)),
         "loads"),
        ("child out of range", edit(lambda d: d["nodes"][0].setdefault(
            "children", []).append(nnodes + 100)), "error"),
        ("node cycle", edit(cycle), "error"),
        ("root listed twice", edit(root_twice), "error"),
        ("deep chain of 40 nodes", edit(lambda d: chain(d, False)),
         "loads"),
        ("shared children on 40 levels", edit(lambda d: chain(d, True)),
         "error"),
        ("matrix of 15 numbers", edit(lambda d: d["nodes"][0].update(
            matrix=[1.0] * 15)), "error"),
        ("fractional accessor count", edit(lambda d: d["accessors"][0].update(
            count=d["accessors"][0]["count"] + 0.5)), "error"),
        ("negative byte offset", edit(lambda d: d["bufferViews"][0].update(
            byteOffset=-16)), "error"),
        ("mesh index 1e30", edit(lambda d: [
            n.update(mesh=1e30) for n in d["nodes"] if "mesh" in n][:1]),
         "error"),
        ("material index -1", edit(
            lambda d: d["meshes"][0]["primitives"][0].update(material=-1)),
         "error"),
    ]


@pytest.mark.timeout(300)
def test_loader_malformed_files_fail_cleanly(tmp_path):
    """One corruption at a time of a valid saved scene: the loader returns
    an error (or loads, where the format allows it) and never crashes or
    runs away; each load runs in its own process, so a crash shows as a
    signal."""
    import json
    import subprocess
    import sys
    src = api.Scene(api.SCENE_SMALL, 1)
    good = tmp_path / "good.gltf"
    src.save_gltf(str(good))
    doc = json.loads(good.read_text())
    binlen = os.path.getsize(str(tmp_path / "good.bin"))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    probe = ("import sys; from nodebleed_b200 import api\n"
             "try:\n    api.Scene.load_gltf(sys.argv[1])\n"
             "except RuntimeError:\n    sys.exit(3)\n")
    for k, (name, fn, want) in enumerate(_corruptions(doc, binlen)):
        d = fn(doc)
        d["buffers"][0]["uri"] = "good.bin"
        path = tmp_path / ("bad%d.gltf" % k)
        path.write_text(json.dumps(d))
        r = subprocess.run([sys.executable, "-c", probe, str(path)],
                           cwd=root, capture_output=True, text=True,
                           timeout=60)
        assert r.returncode in (0, 3), (name, r.returncode, r.stderr[-500:])
        assert r.returncode == (3 if want == "error" else 0), \
            (name, want, r.returncode)
    # a truncated .bin
    (tmp_path / "short.bin").write_bytes(
        (tmp_path / "good.bin").read_bytes()[:binlen // 2])
    d = json.loads(good.read_text())
    d["buffers"][0]["uri"] = "short.bin"
    (tmp_path / "short.gltf").write_text(json.dumps(d))
    with pytest.raises(RuntimeError):
        api.Scene.load_gltf(str(tmp_path / "short.gltf"))
