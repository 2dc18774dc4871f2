"""nodebleed_b200: B200 path-tracing core for nodebleed.

The product is two in-tree native libraries (see build.py):

* ``libnbhost.so``: C host code mirroring nodebleed's own (render-data
  bridge, SAH-binned BVH8 build, seeded synthetic scenes);
* ``libnbgpu.so``: the sm_100a kernels behind the C ABI of
  ``include/rendgpu.h``.

This package is a thin ctypes layer over both for tests and benchmarks; a C
application links the libraries directly.  Loading fails loudly when a
library is missing: there is no CPU fallback.
"""

from .api import (  # noqa: F401
    HostLib, GpuLib, Scene, RenderData, GpuRenderer, BatchRenderer,
    RendgpuError,
    RAY_DTYPE, HIT_DTYPE, host_lib, gpu_lib, SCENE_SMALL, SCENE_SCALE,
    SCENE_BATCH, SCENE_STRESS, SCENE_TINY, SCENE_GLOSSY, MODE_PATH, MODE_PRIMARY, MODE_NRC,
)
