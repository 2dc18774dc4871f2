"""Radiance-cache frames (RENDGPU_MODE_NRC) on the GPU: queries, training
records, online training, and what the trained cache gains over the plain
tracer at equal device time."""

import numpy as np
import pytest

from nodebleed_b200 import api, nrc_eval

pytestmark = pytest.mark.gpu


def test_nrc_frames_produce_queries_and_records(gpu):
    scene = api.Scene(api.SCENE_SMALL, 1)
    rd = api.RenderData(scene, 160, 90, 1)
    gr = api.GpuRenderer(rd, max_depth=5, mode=api.MODE_NRC, seed=3,
                         timing=True, nrc_warmup=2).upload()
    for f in range(6):
        rays = gr.frame()
        st = gr.stats()
        assert rays > 0 and st["device_errors"] == 0
        assert st["nrc_records"] > 0
        # warm-up frames trace every path unbiased: no cache queries
        assert (st["nrc_queries"] == 0) == (f < 2)
    gr.readback(1)
    img = rd.acc()
    assert np.isfinite(img).all() and (img >= 0).all()
    gr.close()


def test_nrc_relmse_reduction_is_reported(gpu):
    """What the trained cache gains: against a 256-spp plain reference, the
    FP64 relMSE of the cache renderer and of the plain tracer at equal
    device time.  On the scale scene at 640x360 (frames large enough that
    launch overhead does not decide the timing) the cache must be ahead,
    and the evaluation must be self-consistent."""
    scene = api.Scene(api.SCENE_SCALE, 1)
    w, h, depth = 640, 360, 8
    ref = nrc_eval.reference(scene, w, h, depth, 256)
    res = nrc_eval.equal_time(scene, w, h, depth, 32, ref)
    print({k: res[k] for k in ("ratio_plain_over_nrc",)}, res["nrc"]["ms"],
          res["plain"]["frames"])
    assert np.isfinite(res["nrc"]["relmse"]) and res["nrc"]["relmse"] > 0
    assert np.isfinite(res["plain"]["relmse"]) and res["plain"]["relmse"] > 0
    assert res["plain"]["ms"] >= res["nrc"]["ms"] or res["plain"]["frames"] == 1
    assert res["ratio_plain_over_nrc"] > 1.1, res
