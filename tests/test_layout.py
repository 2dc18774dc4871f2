"""The C-ABI boundary: struct layout against the reference, exported
symbols of include/rendgpu.h, loading without a GPU."""

import ctypes as C
import os
import re

import pytest

from nodebleed_b200 import api
import oracle_lib as ol

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# sizeof/offsetof the reference compiled from rend.h reports (recorded from
# refh_layout in oracle/ref_harness.c, rend.h:17-147)
REF_LAYOUT = [800, 0, 8, 16, 24, 32, 40, 48, 56, 64, 736, 748, 752, 760, 768,
              776, 780, 784, 788, 672, 64, 640, 256, 192, 64, 48, 48, 32, 32,
              144, 160, 48, 52, 56]


def test_rdata_mirror_matches_recorded_layout():
    R = api.RData
    mine = [C.sizeof(R), R.mtls.offset, R.tris.offset, R.nrms.offset,
            R.instcnt.offset, R.insts.offset, R.aabbs.offset,
            R.bnodes.offset, R.tlasofs.offset, R.cam.offset, R.bgcol.offset,
            R.width.offset, R.height.offset, R.acc.offset, R.buf.offset,
            R.blknum.offset, R.rays.offset, R.spp.offset, R.samples.offset]
    assert mine == REF_LAYOUT[:19]


def test_reference_layout_is_the_recorded_one():
    R = ol.ref()
    if R is None:
        pytest.skip("reference build not present")
    out = (C.c_ulonglong * 64)()
    n = R.refh_layout(out, 64)
    assert list(out[:n]) == REF_LAYOUT


def _header_symbols(path):
    text = open(path).read()
    return sorted(set(re.findall(r"\b(rendgpu_[a-z_]+)\s*\(", text)))


@pytest.mark.parametrize("lang,std", [("c", "-std=c11"),
                                      ("c++", "-std=c++17")])
def test_header_compiles_alone(tmp_path, lang, std):
    """include/rendgpu.h is self-contained C and C++ (what a binding's
    build compiles)."""
    import subprocess
    src = tmp_path / ("t.c" if lang == "c" else "t.cpp")
    src.write_text('#include "rendgpu.h"\nint main(void) { return '
                   'RENDGPU_OK; }\n')
    cc = "gcc" if lang == "c" else "g++"
    r = subprocess.run([cc, std, "-Wall", "-Wextra", "-Werror",
                        "-fsyntax-only", "-I", os.path.join(ROOT, "include"),
                        str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_gpu_library_exports_every_header_symbol():
    syms = _header_symbols(os.path.join(ROOT, "include", "rendgpu.h"))
    assert len(syms) >= 17
    L = api.gpu_lib().L
    for s in syms:
        assert hasattr(L, s), s


def test_host_library_exports_every_header_symbol():
    text = open(os.path.join(ROOT, "nodebleed_b200", "csrc", "host",
                             "nb_host.h")).read()
    syms = sorted(set(re.findall(r"\b(nbh_[a-z0-9_]+)\s*\(", text)))
    L = api.host_lib().L
    for s in syms:
        assert hasattr(L, s), s


def test_gpu_library_has_sm100a_code():
    path = os.path.join(ROOT, "nodebleed_b200", "libnbgpu.so")
    data = open(path, "rb").read()
    assert b"sm_100a" in data


def test_init_without_device_fails_cleanly():
    import conftest
    if conftest.has_gpu():
        pytest.skip("a GPU is present")
    scene = api.Scene(api.SCENE_TINY, 1)
    rd = api.RenderData(scene)
    with pytest.raises(api.RendgpuError) as e:
        api.GpuRenderer(rd)
    assert e.value.code == -7  # RENDGPU_ENODEV
