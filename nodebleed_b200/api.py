"""ctypes bindings of libnbhost.so and libnbgpu.so (include/rendgpu.h)."""

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

SCENE_SMALL, SCENE_SCALE, SCENE_BATCH, SCENE_STRESS, SCENE_TINY = 1, 2, 3, 5, 9
SCENE_GLOSSY = 6
MODE_PATH, MODE_PRIMARY, MODE_NRC = 0, 1, 2
RESOLVE_WRAP, RESOLVE_REINHARD, RESOLVE_ACES = 0, 1, 2
FLAG_TIMING, FLAG_COUNT, FLAG_GRAPH = 1, 2, 4

# struct rendgpu_ray / rendgpu_hit (32 / 16 bytes)
RAY_DTYPE = np.dtype([("o", "<f4", (3,)), ("tmax", "<f4"), ("d", "<f4", (3,)),
                      ("pad", "<u4")])
HIT_DTYPE = np.dtype([("t", "<f4"), ("u", "<f4"), ("v", "<f4"), ("id", "<u4")])

STATUS = {0: "ok", -1: "EINVAL", -2: "ENOMEM", -3: "ECUDA", -4: "ELIMIT",
          -5: "ESTATE", -6: "EDEVICE", -7: "ENODEV"}


class RendgpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"rendgpu {STATUS.get(code, code)}: {msg}")
        self.code = code


def _load(name):
    path = os.path.join(HERE, name)
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is not built; run "
                           "`python -m nodebleed_b200.build`")
    return C.CDLL(path)


class RData(C.Structure):
    """struct rdata (rend.h:119-147), 800 bytes."""
    _fields_ = [
        ("mtls", C.c_void_p), ("tris", C.c_void_p), ("nrms", C.c_void_p),
        ("instcnt", C.c_uint32), ("insts", C.c_void_p),
        ("aabbs", C.c_void_p), ("bnodes", C.c_void_p),
        ("tlasofs", C.c_uint32), ("_pad0", C.c_uint32),
        ("cam", C.c_ubyte * 672), ("bgcol", C.c_float * 3),
        ("width", C.c_uint32), ("height", C.c_uint32),
        ("acc", C.c_void_p), ("buf", C.c_void_p), ("blknum", C.c_int32),
        ("rays", C.c_uint32), ("spp", C.c_uint32), ("samples", C.c_uint32),
        ("_pad1", C.c_ubyte * 8)]


class SceneStruct(C.Structure):
    """struct nbh_scene (nb_host.h)."""
    _fields_ = [
        ("meshcnt", C.c_uint32), ("meshes", C.c_void_p),
        ("mtlcnt", C.c_uint32), ("mtls", C.c_void_p),
        ("instcnt", C.c_uint32), ("insts", C.c_void_p),
        ("cam", C.c_float * 16), ("bgcol", C.c_float * 3),
        ("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32),
        ("depth", C.c_uint32), ("pad", C.c_uint32)]


class RendgpuCfg(C.Structure):
    _fields_ = [("size", C.c_uint32), ("max_depth", C.c_uint32),
                ("mode", C.c_uint32), ("flags", C.c_uint32),
                ("seed", C.c_uint64), ("device", C.c_int32),
                ("block", C.c_uint32), ("sched", C.c_uint32),
                ("reserved", C.c_uint32 * 7)]


class RendgpuStats(C.Structure):
    _fields_ = [("rays", C.c_uint64), ("closest_rays", C.c_uint64),
                ("shadow_rays", C.c_uint64), ("trace_launches", C.c_uint32),
                ("launches", C.c_uint32), ("ms_frame", C.c_float),
                ("ms_trace", C.c_float), ("ms_shadow", C.c_float),
                ("ms_shade", C.c_float), ("device_errors", C.c_uint32),
                ("max_stack", C.c_uint32), ("device_bytes", C.c_uint64),
                ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64),
                ("node_visits", C.c_uint64), ("tri_tests", C.c_uint64),
                ("bounce_closest", C.c_uint32 * 16),
                ("bounce_shadow", C.c_uint32 * 16),
                ("nrc_queries", C.c_uint32), ("nrc_records", C.c_uint32),
                ("ms_nrc", C.c_float), ("nrc_loss", C.c_float)]

    def as_dict(self):
        d = {}
        for k, _ in self._fields_:
            v = getattr(self, k)
            d[k] = list(v) if hasattr(v, "__len__") else v
        return d


class RendgpuTune(C.Structure):
    _fields_ = [("block", C.c_uint32), ("stack", C.c_uint32),
                ("queue", C.c_uint32), ("sched", C.c_uint32),
                ("ms", C.c_float), ("sort", C.c_uint32),
                ("fuse", C.c_uint32), ("force", C.c_uint32)]

    def as_dict(self):
        return {"block": self.block, "stack": self.stack,
                "queue": self.queue, "sched": self.sched, "ms": self.ms,
                "sort": self.sort, "fuse": self.fuse, "force": self.force}

    @classmethod
    def make(cls, block=0, stack=0, queue=0, sched=0, sort=0, fuse=0,
             force=0):
        t = cls()
        t.block, t.stack, t.queue, t.sched = block, stack, queue, sched
        t.sort, t.fuse, t.force = sort, fuse, force
        return t


class RendgpuSceneStats(C.Structure):
    _fields_ = [("closest_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("paths", C.c_uint64), ("pixels", C.c_uint64)]


class HostLib:
    def __init__(self):
        L = _load("libnbhost.so")
        vp, u32, u64 = C.c_void_p, C.c_uint32, C.c_uint64
        L.nbh_scene_gen.argtypes = [vp, C.c_int, u64, u32]
        L.nbh_scene_free.argtypes = [vp]
        L.nbh_scene_tricnt.argtypes = [vp]
        L.nbh_scene_tricnt.restype = u32
        L.nbh_scene_instcnt.argtypes = [vp]
        L.nbh_scene_instcnt.restype = u32
        L.nbh_scene_insttris.argtypes = [vp]
        L.nbh_scene_insttris.restype = C.c_double
        L.nbh_rdata_new.restype = vp
        L.nbh_rdata_delete.argtypes = [vp]
        L.nbh_rend_init.argtypes = [vp, u32, u32, u32, u32]
        L.nbh_rend_release.argtypes = [vp]
        L.nbh_rend_resaccum.argtypes = [vp, u32, u32]
        L.nbh_rend_clraccum.argtypes = [vp]
        L.nbh_cpy_rdata.argtypes = [vp, vp]
        L.nbh_upd_rinsts.argtypes = [vp, vp]
        L.nbh_upd_rcam.argtypes = [vp, vp, C.c_float, C.c_float]
        L.nbh_prepstatic.argtypes = [vp]
        L.nbh_prepdynamic.argtypes = [vp]
        L.nbh_rdata_from_scene.argtypes = [vp, vp]
        L.nbh_scene_load_gltf.argtypes = [vp, C.c_char_p, u32]
        L.nbh_scene_save_gltf.argtypes = [vp, C.c_char_p]
        self.L = L


class GpuLib:
    def __init__(self):
        L = _load("libnbgpu.so")
        vp, u32 = C.c_void_p, C.c_uint32
        for fn, args in [
                ("rendgpu_init", [vp, vp]), ("rendgpu_release", [vp]),
                ("rendgpu_upload_static", [vp]),
                ("rendgpu_upload_dynamic", [vp]),
                ("rendgpu_resaccum", [vp]), ("rendgpu_clraccum", [vp]),
                ("rendgpu_render", [vp]), ("rendgpu_readback", [vp, C.c_int]),
                ("rendgpu_trace_rays", [vp, vp, u32, vp]),
                ("rendgpu_occluded", [vp, vp, u32, vp]),
                ("rendgpu_trace_rays_device", [vp, vp, u32, vp]),
                ("rendgpu_occluded_device", [vp, vp, u32, vp]),
                ("rendgpu_trace_rays_device_noalloc", [vp, vp, u32, vp]),
                ("rendgpu_nrc_reset", [vp, C.c_uint64]),
                ("rendgpu_relmse_device", [vp, vp, vp]),
                ("rendgpu_nrc_weights", [vp, vp, C.c_int]),
                ("rendgpu_nrc_encode_device", [vp, vp, u32, vp]),
                ("rendgpu_nrc_infer_device", [vp, vp, u32, vp]),
                ("rendgpu_nrc_query_device", [vp, vp, u32, vp, u32]),
                ("rendgpu_check_bounded_wait", [vp, u32, vp]),
                ("rendgpu_nrc_train_device", [vp, vp, vp, u32, C.c_int, vp,
                                              vp]),
                ("rendgpu_nrc_train_raw_device", [vp, vp, vp, u32, C.c_int,
                                                  vp, vp, vp]),
                ("rendgpu_nrc_grid", [vp, vp, C.c_int]),
                ("rendgpu_sync", [vp]), ("rendgpu_get_stats", [vp, vp]),
                ("rendgpu_get_lights", [vp, vp, u32, vp]),
                ("rendgpu_capture", [vp, u32, u32]),
                ("rendgpu_tune_save", [vp, C.c_char_p]),
                ("rendgpu_tune_load", [vp, C.c_char_p]),
                ("rendgpu_batch_tune_save", [vp, C.c_char_p]),
                ("rendgpu_batch_tune_load", [vp, C.c_char_p]),
                ("rendgpu_update_instances_device", [vp, vp, u32, u32]),
                ("rendgpu_update_instances", [vp, vp, u32, u32]),
                ("rendgpu_get_instances", [vp, vp, vp, u32, vp]),
                ("rendgpu_blas_host", [vp, u32, u32, vp, u32, vp, u32, vp]),
                ("rendgpu_set_resolve", [vp, u32, C.c_float]),
                ("rendgpu_batch_set_resolve", [vp, u32, C.c_float]),
                ("rendgpu_captured", [vp, u32, vp, vp, vp, vp]),
                ("rendgpu_get_stream", [vp, vp]),
                ("rendgpu_set_tune", [vp, vp]),
                ("rendgpu_get_tune", [vp, vp]),
                ("rendgpu_autotune", [vp, u32, vp, vp, u32, vp]),
                ("rendgpu_batch_init", [vp, u32, vp, vp, vp]),
                ("rendgpu_batch_release", [vp]),
                ("rendgpu_batch_upload_static", [vp]),
                ("rendgpu_batch_upload_dynamic", [vp]),
                ("rendgpu_batch_resaccum", [vp]),
                ("rendgpu_batch_clraccum", [vp]),
                ("rendgpu_batch_render", [vp]),
                ("rendgpu_batch_readback", [vp, C.c_int]),
                ("rendgpu_batch_get_stats", [vp, vp, vp, u32]),
                ("rendgpu_batch_set_tune", [vp, vp]),
                ("rendgpu_batch_get_tune", [vp, vp]),
                ("rendgpu_batch_autotune", [vp, u32, vp, vp, u32, vp]),
                ("rendgpu_batch_get_stream", [vp, vp]),
                ("rendgpu_batch_last_error", [vp]),
                ("rendgpu_last_error", [vp])]:
            f = getattr(L, fn)
            f.argtypes = args
            f.restype = C.c_int
        L.rendgpu_strerror.argtypes = [vp]
        L.rendgpu_strerror.restype = C.c_char_p
        L.rendgpu_batch_strerror.argtypes = [vp]
        L.rendgpu_batch_strerror.restype = C.c_char_p
        self.L = L


_HOST = None
_GPU = None


def host_lib():
    global _HOST
    if _HOST is None:
        _HOST = HostLib()
    return _HOST


def gpu_lib():
    global _GPU
    if _GPU is None:
        _GPU = GpuLib()
    return _GPU


class Scene:
    """A seeded synthetic scene (nbh_scene_gen), or one loaded from glTF
    (Scene.load_gltf)."""

    def __init__(self, family, seed=1, param=0):
        self.h = host_lib().L
        self.s = SceneStruct()
        if family is None:  # filled by load_gltf
            self.family = self.seed = self.param = None
            return
        rc = self.h.nbh_scene_gen(C.byref(self.s), family, seed, param)
        if rc != 0:
            raise RuntimeError(f"nbh_scene_gen({family}, {seed}) = {rc}")
        self.family, self.seed, self.param = family, seed, param

    @classmethod
    def load_gltf(cls, path, extras=True):
        """nbh_scene_load_gltf; extras=False reads the file as nodebleed's
        importer would (no exact-transform extras)."""
        sc = cls(None)
        rc = sc.h.nbh_scene_load_gltf(C.byref(sc.s), os.fsencode(path),
                                      0 if extras else 1)
        if rc != 0:
            raise RuntimeError(f"nbh_scene_load_gltf({path}) = {rc}")
        return sc

    def save_gltf(self, path):
        rc = self.h.nbh_scene_save_gltf(self.ptr, os.fsencode(path))
        if rc != 0:
            raise RuntimeError(f"nbh_scene_save_gltf({path}) = {rc}")

    @property
    def ptr(self):
        return C.addressof(self.s)

    @property
    def tris(self):
        return self.h.nbh_scene_tricnt(self.ptr)

    @property
    def insts(self):
        return self.h.nbh_scene_instcnt(self.ptr)

    @property
    def inst_tris(self):
        return self.h.nbh_scene_insttris(self.ptr)

    def globs(self):
        """Writable (instances, 16) view of every instance's row-major
        object->world matrix (nbh_inst.glob)."""
        n = self.s.instcnt
        raw = (C.c_ubyte * (72 * n)).from_address(self.s.insts)
        return np.ctypeslib.as_array(raw).view(np.float32).reshape(n, 18)[
            :, 2:]

    def settings(self):
        s = self.s
        return dict(width=s.width, height=s.height, spp=s.spp, depth=s.depth)

    def close(self):
        if self.s is not None:
            self.h.nbh_scene_free(self.ptr)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RenderData:
    """A `struct rdata` filled from a scene by the host library (rend_init,
    cpy_rdata, prepstatic, upd_rinsts, prepdynamic, resaccum, upd_rcam)."""

    def __init__(self, scene, width=None, height=None, spp=None):
        self.h = host_lib().L
        self.ptr = self.h.nbh_rdata_new()
        if not self.ptr:
            raise MemoryError("nbh_rdata_new")
        rc = self.h.nbh_rdata_from_scene(self.ptr, scene.ptr)
        if rc != 0:
            raise RuntimeError(f"nbh_rdata_from_scene = {rc}")
        self.scene = scene
        self.buf = None
        self.users = []  # renderers on this rdata, closed with it
        if width or height or spp:
            self.resize(width or self.rd.width, height or self.rd.height,
                        spp or self.rd.spp)
        self.attach_buf()

    @property
    def rd(self):
        return RData.from_address(self.ptr)

    def resize(self, w, h, spp=None):
        if spp is not None:
            self.rd.spp = spp
        self.h.nbh_rend_resaccum(self.ptr, w, h)
        camp = C.addressof(self.scene.s) + SceneStruct.cam.offset
        self.h.nbh_upd_rcam(self.ptr, camp, float(w), float(h))
        self.attach_buf()

    def update_host(self):
        """The reference frame loop's host update after a transform change
        (main.c:257-264): upd_rinsts, then the TLAS build (prepdynamic)."""
        rc = self.h.nbh_upd_rinsts(self.ptr, self.scene.ptr)
        if rc != 0:
            raise RuntimeError("nbh_upd_rinsts: singular transform")
        self.h.nbh_prepdynamic(self.ptr)

    def globinv(self):
        """(instances, 12) world->object 3x4 of rd->insts."""
        n = self.rd.instcnt
        raw = (C.c_ubyte * (64 * n)).from_address(self.rd.insts)
        return np.ctypeslib.as_array(raw).view(np.float32).reshape(n, 16)[
            :, :12].copy()

    def aabbs(self):
        """(instances, 6) world boxes of rd->aabbs (min xyz, max xyz)."""
        n = self.rd.instcnt
        raw = (C.c_ubyte * (32 * n)).from_address(self.rd.aabbs)
        a = np.ctypeslib.as_array(raw).view(np.float32).reshape(n, 8)
        return np.concatenate([a[:, 0:3], a[:, 4:7]], axis=1).copy()

    def attach_buf(self):
        n = self.rd.width * self.rd.height
        self.buf = np.zeros(n, np.uint32)
        self.rd.buf = self.buf.ctypes.data

    def acc(self):
        n = self.rd.width * self.rd.height * 3
        a = (C.c_float * n).from_address(self.rd.acc)
        return np.ctypeslib.as_array(a).reshape(self.rd.height,
                                                self.rd.width, 3)

    def eye(self):
        return np.frombuffer(bytes(self.rd.cam[:12]), np.float32).copy()

    def close(self):
        if self.ptr:
            # a GPU context keyed by this rdata must not outlive it (a new
            # rdata at the same address would find it)
            for u in self.users:
                u.close()
            self.users = []
            self.h.nbh_rend_release(self.ptr)
            self.h.nbh_rdata_delete(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_cfg(max_depth=5, mode=MODE_PATH, seed=1, timing=False, device=0,
             count=False, sched=0, graph=False, block=0):
    cfg = RendgpuCfg()
    cfg.size = C.sizeof(RendgpuCfg)
    cfg.max_depth = max_depth
    cfg.mode = mode
    cfg.flags = (FLAG_TIMING if timing else 0) | \
        (FLAG_COUNT if count else 0) | (FLAG_GRAPH if graph else 0)
    cfg.seed = seed
    cfg.device = device
    cfg.sched = sched
    cfg.block = block
    return cfg


def _autotune(fn, handle, frames, cap, check):
    best = RendgpuTune()
    log = (RendgpuTune * cap)()
    n = C.c_uint32()
    check(fn(handle, frames, C.byref(best), log, cap, C.byref(n)))
    return best.as_dict(), [log[i].as_dict() for i in range(min(n.value,
                                                                 cap))]


class GpuRenderer:
    """The rendgpu C ABI on one RenderData."""

    def __init__(self, rdata, max_depth=5, mode=MODE_PATH, seed=1,
                 timing=False, device=0, count=False, sched=0,
                 nrc_warmup=0, nrc_lr=0.0, graph=False, block=0,
                 nrc_end=0, nrc_steps=0, ref_tlas=False, nrc_grid=True,
                 nrc_train_paths=0, ref_blas=False):
        self.g = gpu_lib().L
        self.rdata = rdata
        self.ptr = rdata.ptr
        cfg = make_cfg(max_depth, mode, seed, timing, device, count, sched,
                       graph, block)
        cfg.reserved[0] = C.c_uint32.from_buffer_copy(
            C.c_float(nrc_lr)).value
        cfg.reserved[1] = nrc_warmup
        cfg.reserved[2] = nrc_end
        cfg.reserved[3] = nrc_steps
        cfg.reserved[4] = (1 if ref_tlas else 0) | (2 if ref_blas else 0)
        cfg.reserved[5] = 0 if nrc_grid else 1
        cfg.reserved[6] = nrc_train_paths
        rc = self.g.rendgpu_init(self.ptr, C.byref(cfg))
        if rc != 0:
            raise RendgpuError(rc, "rendgpu_init")
        self.live = True
        rdata.users.append(self)

    def _ck(self, rc, what):
        if rc != 0:
            raise RendgpuError(rc, f"{what}: "
                               f"{self.g.rendgpu_strerror(self.ptr).decode()}")

    def upload(self):
        self._ck(self.g.rendgpu_upload_static(self.ptr), "upload_static")
        self._ck(self.g.rendgpu_upload_dynamic(self.ptr), "upload_dynamic")
        self._ck(self.g.rendgpu_resaccum(self.ptr), "resaccum")
        return self

    def upload_dynamic(self):
        self._ck(self.g.rendgpu_upload_dynamic(self.ptr), "upload_dynamic")

    def clraccum(self):
        self._ck(self.g.rendgpu_clraccum(self.ptr), "clraccum")

    def frame(self):
        """One frame and main.c's bookkeeping after the join
        (main.c:424-426).  Returns the frame's ray count."""
        rd = self.rdata.rd
        self.g.rendgpu_render(self.ptr)
        self._ck(self.g.rendgpu_last_error(self.ptr), "render")
        st = self.stats()
        rd.blknum = 0
        rd.rays = 0
        rd.samples += rd.spp
        return st["rays"]

    def readback(self, which=3):
        self._ck(self.g.rendgpu_readback(self.ptr, which), "readback")

    def trace(self, rays):
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        hits = np.zeros(len(rays), HIT_DTYPE)
        self._ck(self.g.rendgpu_trace_rays(self.ptr, rays.ctypes.data,
                                           len(rays), hits.ctypes.data),
                 "trace_rays")
        return hits

    def occluded(self, rays):
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        occl = np.zeros(len(rays), np.uint8)
        self._ck(self.g.rendgpu_occluded(self.ptr, rays.ctypes.data,
                                         len(rays), occl.ctypes.data),
                 "occluded")
        return occl

    def stats(self):
        st = RendgpuStats()
        self._ck(self.g.rendgpu_get_stats(self.ptr, C.byref(st)), "stats")
        return st.as_dict()

    def set_tune(self, **kw):
        t = RendgpuTune.make(**kw)
        self._ck(self.g.rendgpu_set_tune(self.ptr, C.byref(t)), "set_tune")

    def get_tune(self):
        t = RendgpuTune()
        self._ck(self.g.rendgpu_get_tune(self.ptr, C.byref(t)), "get_tune")
        return t.as_dict()

    def autotune(self, frames=2, cap=64):
        """Returns (best setting, every measured setting)."""
        return _autotune(self.g.rendgpu_autotune, self.ptr, frames, cap,
                         lambda rc: self._ck(rc, "autotune"))

    def tune_save(self, path):
        self._ck(self.g.rendgpu_tune_save(self.ptr, os.fsencode(path)),
                 "tune_save")

    def tune_load(self, path):
        """1 when a stored setting was applied, 0 when none matched."""
        rc = self.g.rendgpu_tune_load(self.ptr, os.fsencode(path))
        if rc < 0:
            self._ck(rc, "tune_load")
        return rc

    # ---- neural radiance cache
    NRC_PARAMS = 5 * 4096 + 8 * 64

    def nrc_reset(self, seed=1):
        self._ck(self.g.rendgpu_nrc_reset(self.ptr, seed), "nrc_reset")

    def nrc_weights(self, w=None):
        """Get (w is None) or set the FP32 master weights."""
        if w is None:
            out = np.zeros(self.NRC_PARAMS, np.float32)
            self._ck(self.g.rendgpu_nrc_weights(self.ptr, out.ctypes.data, 0),
                     "nrc_weights")
            return out
        w = np.ascontiguousarray(w, np.float32)
        self._ck(self.g.rendgpu_nrc_weights(self.ptr, w.ctypes.data, 1),
                 "nrc_weights")

    NRC_GRID_PARAMS = 8 * 131072 * 2

    def nrc_grid(self, t=None):
        """Get (t is None) or set the hash grid's FP32 table."""
        if t is None:
            out = np.zeros(self.NRC_GRID_PARAMS, np.float32)
            self._ck(self.g.rendgpu_nrc_grid(self.ptr, out.ctypes.data, 0),
                     "nrc_grid")
            return out
        t = np.ascontiguousarray(t, np.float32)
        self._ck(self.g.rendgpu_nrc_grid(self.ptr, t.ctypes.data, 1),
                 "nrc_grid")

    def relmse(self, ref_device_ptr):
        """relMSE of the accumulated image against a device reference
        image (W*H*3 floats), reduced in FP64 on the device."""
        out = C.c_double()
        self._ck(self.g.rendgpu_relmse_device(self.ptr, ref_device_ptr,
                                              C.byref(out)), "relmse")
        return out.value

    def stream(self):
        """cudaStream_t of this context, as an integer handle."""
        h = C.c_void_p()
        self._ck(self.g.rendgpu_get_stream(self.ptr, C.byref(h)), "stream")
        return h.value or 0

    def lights(self):
        area = C.c_float()
        n = self.g.rendgpu_get_lights(self.ptr, None, 0, C.byref(area))
        if n < 0:
            self._ck(n, "get_lights")
        out = np.zeros((max(n, 1), 20), np.float32)
        self.g.rendgpu_get_lights(self.ptr, out.ctypes.data, n, C.byref(area))
        return out[:n], area.value

    def set_resolve(self, op=0, exposure=1.0):
        """8-bit resolve: 0 the reference's wrapping pack, 1 Reinhard,
        2 ACES (with exposure and the sRGB transfer function)."""
        self._ck(self.g.rendgpu_set_resolve(self.ptr, op, exposure),
                 "set_resolve")

    def update_instances(self, globs, refit=False, tight=False,
                         collapse=None):
        """Device-side scene update from (instances, 16) object->world
        matrices (host array: copied; else an integer device pointer).
        collapse: None = the library's choice by instance count, True =
        the collapsed one-CTA TLAS build, False = level by level."""
        n = self.rdata.rd.instcnt
        flags = (1 if refit else 0) | (2 if tight else 0) | \
            (0 if collapse is None else (4 if collapse else 8))
        if isinstance(globs, int):
            self._ck(self.g.rendgpu_update_instances_device(self.ptr, globs,
                                                            n, flags),
                     "update_instances_device")
        else:
            g = np.ascontiguousarray(globs, np.float32)
            assert g.shape == (n, 16)
            self._ck(self.g.rendgpu_update_instances(self.ptr,
                                                     g.ctypes.data, n, flags),
                     "update_instances")

    def instances(self, boxes=True):
        """(world->object 3x4 (n, 12), world boxes (n, 6) or None, TLAS
        info (nodes, depth, overflow) or None) held by the device."""
        n = self.rdata.rd.instcnt
        xf = np.zeros((n, 12), np.float32)
        wb = np.zeros((n, 6), np.float32) if boxes else None
        info = (C.c_uint32 * 3)()
        rc = self.g.rendgpu_get_instances(
            self.ptr, xf.ctypes.data, wb.ctypes.data if boxes else None, n,
            info if boxes else None)
        if rc < 0:
            self._ck(rc, "get_instances")
        return xf, wb, (tuple(info) if boxes else None)

    def capture(self, bounces, cap):
        """Record, in every later frame, up to `cap` closest-hit rays (with
        the frame's hits) and shadow rays of each bounce in `bounces`."""
        mask = 0
        for k in bounces:
            mask |= 1 << k
        self._ck(self.g.rendgpu_capture(self.ptr, mask, cap if mask else 0),
                 "capture")
        self.cap = cap

    def captured(self, bounce):
        """(rays, hits, shadow rays, counts) of the last frame's capture of
        `bounce`; counts = (returned, traced, shadow returned, shadow
        generated)."""
        cap = self.cap
        rays = np.zeros(cap, RAY_DTYPE)
        hits = np.zeros(cap, HIT_DTYPE)
        shadow = np.zeros(cap, RAY_DTYPE)
        counts = (C.c_uint32 * 4)()
        self._ck(self.g.rendgpu_captured(self.ptr, bounce, rays.ctypes.data,
                                         hits.ctypes.data, shadow.ctypes.data,
                                         counts), "captured")
        n, ns = counts[0], counts[2]
        return rays[:n], hits[:n], shadow[:ns], tuple(counts)

    def close(self):
        if self.live:
            self.g.rendgpu_release(self.ptr)
            self.live = False

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchRenderer:
    """rendgpu_batch_*: several RenderData rendered by one captured launch
    sequence over shared ray queues.  max_depth: one value for all scenes
    or one per scene."""

    def __init__(self, rdatas, max_depth=5, mode=MODE_PATH, seed=1,
                 timing=False, device=0, sched=0, block=0, nrc_grid=True,
                 ref_blas=False):
        self.g = gpu_lib().L
        self.rdatas = list(rdatas)
        n = len(self.rdatas)
        depths = max_depth if hasattr(max_depth, "__len__") else \
            [max_depth] * n
        self.depths = (C.c_uint32 * n)(*depths)
        ptrs = (C.c_void_p * n)(*[r.ptr for r in self.rdatas])
        cfg = make_cfg(max(depths), mode, seed, timing, device, False, sched,
                       True, block)
        cfg.reserved[4] = 2 if ref_blas else 0
        cfg.reserved[5] = 0 if nrc_grid else 1
        h = C.c_void_p()
        rc = self.g.rendgpu_batch_init(ptrs, n, self.depths, C.byref(cfg),
                                       C.byref(h))
        if rc != 0:
            raise RendgpuError(rc, "rendgpu_batch_init")
        self.h = h.value
        self.live = True
        for r in self.rdatas:
            r.users.append(self)

    def _ck(self, rc, what):
        if rc != 0:
            raise RendgpuError(rc, f"{what}: "
                               f"{self.g.rendgpu_batch_strerror(self.h).decode()}")

    def upload(self):
        self._ck(self.g.rendgpu_batch_upload_static(self.h), "upload_static")
        self._ck(self.g.rendgpu_batch_upload_dynamic(self.h),
                 "upload_dynamic")
        self._ck(self.g.rendgpu_batch_resaccum(self.h), "resaccum")
        return self

    def clraccum(self):
        self._ck(self.g.rendgpu_batch_clraccum(self.h), "clraccum")

    def frame(self):
        """One frame of every scene, then main.c's bookkeeping on each
        rdata.  Returns the frame's ray count over all scenes."""
        self._ck(self.g.rendgpu_batch_render(self.h), "render")
        total, _ = self.stats()
        for r in self.rdatas:
            rd = r.rd
            rd.blknum = 0
            rd.rays = 0
            rd.samples += rd.spp
        return total["rays"]

    def readback(self, which=3):
        self._ck(self.g.rendgpu_batch_readback(self.h, which), "readback")

    def stats(self):
        """(totals as GpuRenderer.stats, [per-scene counts])."""
        n = len(self.rdatas)
        st = RendgpuStats()
        per = (RendgpuSceneStats * n)()
        self._ck(self.g.rendgpu_batch_get_stats(self.h, C.byref(st), per, n),
                 "stats")
        return st.as_dict(), [{k: getattr(p, k) for k, _ in p._fields_}
                              for p in per]

    def set_tune(self, **kw):
        t = RendgpuTune.make(**kw)
        self._ck(self.g.rendgpu_batch_set_tune(self.h, C.byref(t)),
                 "set_tune")

    def get_tune(self):
        t = RendgpuTune()
        self._ck(self.g.rendgpu_batch_get_tune(self.h, C.byref(t)),
                 "get_tune")
        return t.as_dict()

    def autotune(self, frames=2, cap=64):
        return _autotune(self.g.rendgpu_batch_autotune, self.h, frames, cap,
                         lambda rc: self._ck(rc, "autotune"))

    def tune_save(self, path):
        self._ck(self.g.rendgpu_batch_tune_save(self.h, os.fsencode(path)),
                 "tune_save")

    def tune_load(self, path):
        rc = self.g.rendgpu_batch_tune_load(self.h, os.fsencode(path))
        if rc < 0:
            self._ck(rc, "tune_load")
        return rc

    def stream(self):
        s = C.c_void_p()
        self._ck(self.g.rendgpu_batch_get_stream(self.h, C.byref(s)),
                 "stream")
        return s.value or 0

    def close(self):
        if self.live:
            self.g.rendgpu_batch_release(self.h)
            self.live = False

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
