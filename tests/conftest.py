import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _ensure_built():
    """Build the native libraries if this checkout has none yet (the GPU
    box receives them prebuilt)."""
    from nodebleed_b200 import build as nbuild
    pkg = os.path.join(ROOT, "nodebleed_b200")
    if not os.path.exists(os.path.join(pkg, "libnbhost.so")):
        nbuild.build_host()
    if not os.path.exists(os.path.join(pkg, "libnbgpu.so")):
        nbuild.build_gpu()
    orc = os.path.join(ROOT, "oracle")
    if not os.path.exists(os.path.join(orc, "liboracle.so")):
        subprocess.run(["make", "-C", orc, "liboracle.so"], check=True)
    # the reference itself: built where its sources are named by
    # NODEBLEED_REF; a checkout that travels prebuilt keeps oracle/_ref
    ref_src = os.environ.get("NODEBLEED_REF", "")
    if not os.path.exists(os.path.join(orc, "_ref", "libnbref.so")) and \
            ref_src and os.path.exists(os.path.join(ref_src, "rend.c")):
        subprocess.run(["make", "-C", orc, "ref", "REF=" + ref_src],
                       check=True)


_ensure_built()


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not has_gpu():
        pytest.fail("CUDA device required for a gpu-marked test")
    return True
