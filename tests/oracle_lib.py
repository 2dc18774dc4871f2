"""ctypes access to the CPU checkers under oracle/ (test infrastructure).

* ``oracle/liboracle.so``: the plain-C restatement (oracle/oracle.h);
* ``oracle/_ref/libnbref.so``: the reference renderer compiled from its own
  sources plus a headless driver (oracle/ref_harness.c).

Both are built by ``make -C oracle``.
"""

import ctypes as C
import os

import numpy as np

from nodebleed_b200.api import HIT_DTYPE, RAY_DTYPE

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE = os.path.join(ROOT, "oracle", "liboracle.so")
REF = os.path.join(ROOT, "oracle", "_ref", "libnbref.so")

FLT_MAX = np.float32(np.finfo(np.float32).max)


class Counts(C.Structure):
    _fields_ = [("nodes", C.c_uint64), ("leaves", C.c_uint64),
                ("insts", C.c_uint64), ("rays", C.c_uint64)]


class PtCfg(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("depth", C.c_uint32),
                ("mode", C.c_uint32), ("nthreads", C.c_int),
                ("nlights", C.c_uint32), ("lights", C.c_void_p),
                ("light_area", C.c_float), ("x0", C.c_uint32),
                ("y0", C.c_uint32), ("x1", C.c_uint32), ("y1", C.c_uint32),
                ("closest", C.c_void_p), ("any", C.c_void_p),
                ("counts", C.c_void_p)]


_ORC = None
_REF = None


def oracle():
    global _ORC
    if _ORC is None:
        L = C.CDLL(ORACLE)
        vp, u32 = C.c_void_p, C.c_uint32
        L.orc_trace.argtypes = [vp, vp, u32, vp, vp, C.c_int]
        L.orc_occluded.argtypes = [vp, vp, u32, vp, C.c_int]
        L.orc_refine.argtypes = [vp, vp, u32, vp]
        L.orc_reintersect_f64.argtypes = [vp, vp, vp, u32, vp, vp]
        L.orc_render.argtypes = [vp, vp, vp]
        L.orc_render.restype = C.c_uint64
        L.orc_accumulate.argtypes = [vp, vp]
        L.orc_pcg_first.argtypes = [C.c_uint64, u32, C.c_uint64, u32, vp]
        L.orc_sincos2pi.argtypes = [C.c_float, vp, vp]
        L.orc_mt_bounds.argtypes = [vp, vp, vp, u32, vp]
        L.orc_bruteforce_f64.argtypes = [vp, vp, u32, vp, vp]
        L.orc_ggx_sample.argtypes = [vp, vp, C.c_float, vp, C.c_float,
                                     C.c_float, vp, vp]
        L.orc_ggx_sample.restype = C.c_int
        L.orc_ggx_eval.argtypes = [vp, vp, vp, C.c_float, vp, vp]
        _ORC = L
    return _ORC


def ref():
    global _REF
    if _REF is None:
        if not os.path.exists(REF):
            return None
        L = C.CDLL(REF)
        vp, u32 = C.c_void_p, C.c_uint32
        L.refh_layout.argtypes = [vp, C.c_int]
        L.refh_render_frame.argtypes = [vp, C.c_int]
        L.refh_render_frame.restype = u32
        L.refh_trace.argtypes = [vp, vp, u32, vp, C.c_int]
        L.refh_trace_pckts.argtypes = [vp, vp, u32, vp, C.c_int]
        L.refh_occluded.argtypes = [vp, vp, u32, vp, C.c_int]
        L.refh_camrays.argtypes = [vp, u32, u32, C.c_uint64, C.c_uint64,
                                   u32, vp, vp]
        L.rend_staticinit.argtypes = [u32, u32]
        L.rend_prepstatic.argtypes = [vp]
        L.rend_prepdynamic.argtypes = [vp]
        L.rend_staticinit(16, 8)
        _REF = L
    return _REF


class RefRenderData:
    """A struct rdata built entirely by the reference's own host code from a
    glTF file (refh_gltf_rdata): its importer, BVH builds, matrix inverse
    and camera constants.  Offers what GpuRenderer and the oracle read from
    an api.RenderData (ptr, rd, acc, users, close)."""

    def __init__(self, path, w, h, spp):
        from nodebleed_b200 import api
        R = ref()
        if R is None:
            raise RuntimeError("reference build not present")
        R.refh_gltf_rdata.restype = C.c_void_p
        R.refh_gltf_rdata.argtypes = [C.c_char_p, C.c_uint32, C.c_uint32,
                                      C.c_uint32]
        R.refh_rdata_free.argtypes = [C.c_void_p]
        self._R, self._api = R, api
        self.ptr = R.refh_gltf_rdata(os.fsencode(path), w, h, spp)
        if not self.ptr:
            raise RuntimeError("refh_gltf_rdata failed")
        self.users = []
        self.buf = np.zeros(w * h, np.uint32)
        self.rd.buf = self.buf.ctypes.data

    @property
    def rd(self):
        return self._api.RData.from_address(self.ptr)

    def acc(self):
        r = self.rd
        a = (C.c_float * (r.width * r.height * 3)).from_address(r.acc)
        return np.ctypeslib.as_array(a).reshape(r.height, r.width, 3)

    def close(self):
        if self.ptr:
            for u in self.users:
                u.close()
            self.users = []
            self._R.refh_rdata_free(self.ptr)
            self.ptr = None


def ggx_sample(n, wo, alpha, f0, r0, r1):
    """(ok, wi, weight) of the oracle's GGX sampling step."""
    f = lambda v: np.ascontiguousarray(v, np.float32)
    n, wo, f0 = f(n), f(wo), f(f0)
    wi, w = np.zeros(3, np.float32), np.zeros(3, np.float32)
    ok = oracle().orc_ggx_sample(n.ctypes.data, wo.ctypes.data, alpha,
                                 f0.ctypes.data, r0, r1, wi.ctypes.data,
                                 w.ctypes.data)
    return ok, wi, w


def ggx_eval(n, wo, wi, alpha, f0):
    f = lambda v: np.ascontiguousarray(v, np.float32)
    n, wo, wi, f0 = f(n), f(wo), f(wi), f(f0)
    out = np.zeros(3, np.float32)
    oracle().orc_ggx_eval(n.ctypes.data, wo.ctypes.data, wi.ctypes.data,
                          alpha, f0.ctypes.data, out.ctypes.data)
    return out


def fn_addr(lib, name):
    return C.cast(getattr(lib, name), C.c_void_p).value


def ncpu():
    return os.cpu_count() or 1


def orc_trace(rd_ptr, rays, counts=False, nthreads=None):
    L = oracle()
    rays = np.ascontiguousarray(rays, RAY_DTYPE)
    hits = np.zeros(len(rays), HIT_DTYPE)
    cnt = Counts()
    L.orc_trace(rd_ptr, rays.ctypes.data, len(rays), hits.ctypes.data,
                C.byref(cnt) if counts else None, nthreads or ncpu())
    return (hits, cnt) if counts else hits


def orc_refine(rd_ptr, rays, hits):
    rays = np.ascontiguousarray(rays, RAY_DTYPE)
    hits = hits.copy()
    oracle().orc_refine(rd_ptr, rays.ctypes.data, len(rays), hits.ctypes.data)
    return hits


def orc_occluded(rd_ptr, rays, nthreads=None):
    rays = np.ascontiguousarray(rays, RAY_DTYPE)
    out = np.zeros(len(rays), np.uint8)
    oracle().orc_occluded(rd_ptr, rays.ctypes.data, len(rays),
                          out.ctypes.data, nthreads or ncpu())
    return out


def reintersect(rd_ptr, rays, ids):
    rays = np.ascontiguousarray(rays, RAY_DTYPE)
    ids = np.ascontiguousarray(ids, np.uint32)
    t = np.zeros(len(rays))
    b = np.zeros((len(rays), 3))
    oracle().orc_reintersect_f64(rd_ptr, rays.ctypes.data, ids.ctypes.data,
                                 len(rays), t.ctypes.data, b.ctypes.data)
    return t, b


def ref_trace(rd_ptr, rays, packets=False, nthreads=None):
    L = ref()
    rays = np.ascontiguousarray(rays, RAY_DTYPE)
    hits = np.zeros(len(rays), HIT_DTYPE)
    f = L.refh_trace_pckts if packets else L.refh_trace
    f(rd_ptr, rays.ctypes.data, len(rays), hits.ctypes.data,
      nthreads or ncpu())
    return hits


def ref_occluded(rd_ptr, rays, nthreads=None):
    rays = np.ascontiguousarray(rays, RAY_DTYPE)
    out = np.zeros(len(rays), np.uint8)
    ref().refh_occluded(rd_ptr, rays.ctypes.data, len(rays), out.ctypes.data,
                        nthreads or ncpu())
    return out


def orc_render(rd, lights, light_area, depth, mode=0, seed=1, window=None,
               nthreads=None, use_ref=False, counts=None):
    """Frame radiance (H, W, 3) of the oracle path tracer; traversal by the
    restatement or, with use_ref, by the compiled reference."""
    L = oracle()
    r = rd.rd
    W, H = r.width, r.height
    cfg = PtCfg()
    cfg.seed = seed
    cfg.depth = depth
    cfg.mode = mode
    cfg.nthreads = nthreads or ncpu()
    lights = np.ascontiguousarray(lights, np.float32)
    cfg.nlights = len(lights)
    cfg.lights = lights.ctypes.data if len(lights) else None
    cfg.light_area = light_area
    x0, y0, x1, y1 = window or (0, 0, W, H)
    cfg.x0, cfg.y0, cfg.x1, cfg.y1 = x0, y0, x1, y1
    if use_ref:
        R = ref()
        cfg.closest = fn_addr(R, "intersect_tlas")
        cfg.any = fn_addr(R, "intersect_any_tlas")
    if counts is not None:
        cfg.counts = C.addressof(counts)
    rad = np.zeros((H, W, 3), np.float32)
    rays = L.orc_render(rd.ptr, C.byref(cfg), rad.ctypes.data)
    return rad, rays


def mt_bounds(rd_ptr, rays, ids):
    """Forward error bounds (du, dv, dt) of FP32 Moeller-Trumbore for the
    given (ray, triangle) pairs (orc_mt_bounds)."""
    rays = np.ascontiguousarray(rays, RAY_DTYPE)
    ids = np.ascontiguousarray(ids, np.uint32)
    out = np.zeros((len(rays), 3))
    oracle().orc_mt_bounds(rd_ptr, rays.ctypes.data, ids.ctypes.data,
                           len(rays), out.ctypes.data)
    return out


def bruteforce(rd_ptr, rays):
    """FP64 closest hit over every triangle of every entered instance."""
    rays = np.ascontiguousarray(rays, RAY_DTYPE)
    ids = np.zeros(len(rays), np.uint32)
    t = np.zeros(len(rays))
    oracle().orc_bruteforce_f64(rd_ptr, rays.ctypes.data, len(rays),
                                ids.ctypes.data, t.ctypes.data)
    return ids, t


def classify(rd_ptr, rays, ha, hb, eps_t, eps_b, eps_origin=0.0):
    """Compare two hit sets on the same rays.  Returns (n_same, ties,
    bad).  A disagreement is a tie when an FP64 re-intersection of both
    candidates shows either

    * the two within eps_t relative in t (plus the FP32 Moeller-Trumbore
      error bounds of both), or
    * a candidate within eps_b (plus its Moeller-Trumbore error bound) of
      an edge, or outside by less.

    * (eps_origin > 0) a candidate within eps_origin of the ray's origin:
      the zone the renderer's own origin offset (EPS2, util.h:8) exists to
      keep rays out of, where which implementation sees a surface is
      decided by the rounding of its world->object transform.

    The Moeller-Trumbore bounds cover the reference's and the oracle's own
    evaluation of the test; eps_t/eps_b cover the reference's rcpps."""
    miss_a = ha["t"] == FLT_MAX
    miss_b = hb["t"] == FLT_MAX
    same = (miss_a & miss_b) | (~miss_a & ~miss_b & (ha["id"] == hb["id"]))
    idx = np.nonzero(~same)[0]
    ties, bad = [], []
    if len(idx):
        r = rays[idx]
        ta, ba = reintersect(rd_ptr, r, ha["id"][idx])
        tb, bb = reintersect(rd_ptr, r, hb["id"][idx])
        ea = mt_bounds(rd_ptr, r, ha["id"][idx])
        eb = mt_bounds(rd_ptr, r, hb["id"][idx])

        def near(b, e):
            return (b[1] < eps_b + e[0] or b[2] < eps_b + e[1] or
                    b[0] < eps_b + e[0] + e[1])
        for j, i in enumerate(idx):
            near_a = (not miss_a[i]) and near(ba[j], ea[j])
            near_b = (not miss_b[i]) and near(bb[j], eb[j])
            close_t = (not miss_a[i] and not miss_b[i] and
                       abs(ta[j] - tb[j]) <= eps_t * min(abs(ta[j]),
                                                         abs(tb[j])) +
                       ea[j][2] + eb[j][2])
            at_origin = ((not miss_a[i] and abs(ta[j]) < eps_origin) or
                         (not miss_b[i] and abs(tb[j]) < eps_origin))
            if near_a or near_b or close_t or at_origin:
                ties.append(i)
            else:
                bad.append(i)
    return int(same.sum()), ties, bad


def agrees_with_truth(rd_ptr, rays, hits, rel=1e-6):
    """For each ray: does `hits` hold a closest hit as close as the FP64
    brute-force one (same triangle, or FP64 t within `rel`), or miss where
    the truth's triangle is hit within `rel` of an edge?"""
    tid, tt = bruteforce(rd_ptr, rays)
    ok = np.zeros(len(rays), bool)
    th, bh = reintersect(rd_ptr, rays, hits["id"])
    _, btruth = reintersect(rd_ptr, rays, tid)
    for i in range(len(rays)):
        truth_miss = not np.isfinite(tt[i])
        hit_miss = hits["t"][i] == FLT_MAX
        if truth_miss and hit_miss:
            ok[i] = True
        elif hit_miss:
            ok[i] = np.min(btruth[i]) < rel
        elif truth_miss:
            ok[i] = np.min(bh[i]) > -rel and False
        else:
            ok[i] = (hits["id"][i] == tid[i] or
                     abs(th[i] - tt[i]) <= rel * abs(tt[i]) or
                     np.min(btruth[i]) < rel)
    return ok


def random_rays(rd, n, seed=0, spread=8.0):
    """Half camera-origin rays, half from random interior points; random
    directions."""
    rng = np.random.default_rng(seed)
    eye = rd.eye()
    rays = np.zeros(n, RAY_DTYPE)
    org = rng.uniform(-spread, spread, (n, 3)).astype(np.float32)
    cam = rng.random(n) < 0.5
    org[cam] = eye
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays["o"] = org
    rays["d"] = d.astype(np.float32)
    rays["tmax"] = FLT_MAX
    return rays


def camera_rays(rd, n_side=None, seed=3):
    """Rays through jittered pixel positions of the scene camera (a
    numpy version of the pinhole model, for test ray sets)."""
    r = rd.rd
    cam = np.frombuffer(bytes(r.cam), np.float32)
    eye, ri, up, fwd = cam[0:3], cam[4:7], cam[8:11], cam[12:15]
    W, H = r.width, r.height
    rng = np.random.default_rng(seed)
    ys, xs = np.mgrid[0:H, 0:W]
    xs = xs.ravel() + rng.random(W * H)
    ys = ys.ravel() + rng.random(W * H)
    fov = cam[16 + 8 * 16]  # fovfdist8[0]
    aspect = cam[16 + 8 * 14]
    fd = cam[16 + 8 * 15]
    sx = (xs / W - 0.5) * fov * aspect
    sy = (ys / H - 0.5) * fov
    d = fwd[None] * fd + ri[None] * sx[:, None] - up[None] * sy[:, None]
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.zeros(W * H, RAY_DTYPE)
    rays["o"] = eye
    rays["d"] = d.astype(np.float32)
    rays["tmax"] = FLT_MAX
    return rays


def classify_occlusion(rd_ptr, rays, occ_a, occ_b, blk_a, blk_b, eps_t,
                       eps_b):
    """Compare two occlusion answers on the same shadow rays.  blk_a / blk_b
    are each side's closest hit within the ray's tmax (the blocker it sees;
    t = FLT_MAX when none).  Returns (n_same, ties, bad).  A disagreement is a
    tie when the blocker of the side that reports the ray occluded lies, by
    an FP64 re-intersection with the FP32 object-space ray, within eps_b (plus
    its Moeller-Trumbore bound) of an edge, or within eps_t relative (plus
    the bound) of either end of the segment (0, tmax)."""
    occ_a = np.asarray(occ_a).astype(bool)
    occ_b = np.asarray(occ_b).astype(bool)
    idx = np.nonzero(occ_a != occ_b)[0]
    ties, bad = [], []
    if len(idx):
        r = rays[idx]
        blk = np.where(occ_a[idx], blk_a["id"][idx], blk_b["id"][idx])
        bt = np.where(occ_a[idx], blk_a["t"][idx], blk_b["t"][idx])
        t64, b64 = reintersect(rd_ptr, r, blk)
        e = mt_bounds(rd_ptr, r, blk)
        for j, i in enumerate(idx):
            if bt[j] == FLT_MAX:
                bad.append(i)  # occluded, yet no blocker within tmax
                continue
            tmax = float(rays["tmax"][i])
            near_edge = (b64[j][1] < eps_b + e[j][0] or
                         b64[j][2] < eps_b + e[j][1] or
                         b64[j][0] < eps_b + e[j][0] + e[j][1])
            near_end = (abs(t64[j] - tmax) <= eps_t * tmax + e[j][2] or
                        abs(t64[j]) <= eps_t * tmax + e[j][2])
            (ties if near_edge or near_end else bad).append(i)
    return int((occ_a == occ_b).sum()), ties, bad
