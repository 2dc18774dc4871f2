"""Batched multi-scene frames (rendgpu_batch_*): every scene of a batch
renders bit-identical to the same scene rendered alone; waves, block sizes,
stack depths and graph replay change no bits; the autotuner returns a
setting it measured."""

import numpy as np
import pytest

from nodebleed_b200 import api

pytestmark = pytest.mark.gpu

# (family, scene seed, width, height, spp, max depth): uneven sizes,
# sample counts and depths, as a batch of the 16-scene workload has
SCENES = [(api.SCENE_TINY, 1, 64, 48, 1, 3),
          (api.SCENE_SMALL, 1, 160, 90, 4, 5),
          (api.SCENE_TINY, 2, 96, 72, 2, 8),
          (api.SCENE_SMALL, 3, 120, 68, 1, 12),
          (api.SCENE_GLOSSY, 1, 80, 48, 2, 6)]


def _rdatas(scenes=SCENES):
    out = []
    for fam, seed, w, h, spp, _ in scenes:
        sc = api.Scene(fam, seed)
        out.append(api.RenderData(sc, w, h, spp))
    return out


def _alone(seed=7, frames=2, scenes=SCENES, **kw):
    imgs, rays = [], []
    for rd, (_, _, _, _, _, depth) in zip(_rdatas(scenes), scenes):
        gr = api.GpuRenderer(rd, max_depth=depth, seed=seed, **kw).upload()
        r = []
        for _ in range(frames):
            gr.frame()
            st = gr.stats()
            r.append((st["closest_rays"], st["shadow_rays"]))
        gr.readback(1)
        imgs.append(rd.acc().copy())
        rays.append(r)
        gr.close()
    return imgs, rays


def _batch(seed=7, frames=2, scenes=SCENES, tune=None):
    rds = _rdatas(scenes)
    b = api.BatchRenderer(rds, max_depth=[s[5] for s in scenes],
                          seed=seed).upload()
    if tune:
        b.set_tune(**tune)
    rays = []
    for _ in range(frames):
        b.frame()
        tot, per = b.stats()
        assert tot["device_errors"] == 0
        rays.append([(p["closest_rays"], p["shadow_rays"]) for p in per])
    b.readback(1)
    imgs = [rd.acc().copy() for rd in rds]
    b.close()
    return imgs, rays


@pytest.fixture(scope="module")
def alone(gpu):
    return _alone()


@pytest.fixture(scope="module")
def batched(gpu):
    return _batch()


def test_batch_images_match_scenes_rendered_alone(alone, batched):
    for i, (a, b) in enumerate(zip(alone[0], batched[0])):
        assert a.shape == b.shape
        assert np.array_equal(a, b), (i, np.abs(a - b).max())
        assert a.max() > 0


def test_batch_per_scene_ray_counts(alone, batched):
    for f in range(2):
        for i in range(len(SCENES)):
            assert tuple(batched[1][f][i]) == tuple(alone[1][i][f])


@pytest.mark.parametrize("tune", [
    {"queue": 4096}, {"queue": 20000}, {"block": 64}, {"block": 256},
    {"stack": 32}, {"stack": 48}])
def test_tuning_changes_no_bits(batched, tune):
    imgs, rays = _batch(tune=tune)
    for a, b in zip(batched[0], imgs):
        assert np.array_equal(a, b), tune
    assert rays == batched[1]


def test_graph_replay_matches_direct_launches(gpu):
    scenes = SCENES[1:2]
    direct, _ = _alone(frames=3, scenes=scenes)
    graph, _ = _alone(frames=3, scenes=scenes, graph=True)
    assert np.array_equal(direct[0], graph[0])


def test_autotune_returns_a_measured_setting(gpu):
    rds = _rdatas(SCENES[:2])
    b = api.BatchRenderer(rds, max_depth=[3, 5], timing=True).upload()
    best, log = b.autotune(frames=1)
    assert len(log) >= 6
    assert best["ms"] > 0 and best["ms"] == min(x["ms"] for x in log)
    assert any(all(x[k] == best[k] for k in ("block", "stack", "queue",
                                             "sched")) for x in log)
    got = b.get_tune()
    assert all(got[k] == best[k] for k in ("block", "stack", "queue",
                                           "sched"))
    # the accumulator is cleared; frames render normally afterwards
    b.readback(1)
    assert all(rd.acc().max() == 0 for rd in rds)
    b.frame()
    b.readback(1)
    assert all(rd.acc().max() > 0 for rd in rds)
    b.close()


def test_tuned_setting_persists(gpu, tmp_path):
    """rendgpu_(batch_)tune_save / _load: the tuned setting of a GPU model
    and scene signature comes back in a later context of the same scenes,
    and only there."""
    keys = ("block", "stack", "queue", "sched", "sort", "fuse")
    path = str(tmp_path / "tune.txt")
    b = api.BatchRenderer(_rdatas(SCENES[:2]), max_depth=[3, 5],
                          timing=True).upload()
    best, _ = b.autotune(frames=1)
    b.tune_save(path)
    b.close()
    b2 = api.BatchRenderer(_rdatas(SCENES[:2]), max_depth=[3, 5]).upload()
    assert b2.tune_load(path) == 1
    got = b2.get_tune()
    assert all(got[k] == b2.get_tune()[k] for k in keys)
    assert all(got[k] == best[k] for k in ("block", "stack", "queue",
                                           "sched", "fuse"))
    b2.close()
    b3 = api.BatchRenderer(_rdatas(SCENES[:1]), max_depth=[3]).upload()
    assert b3.tune_load(path) == 0  # another signature
    b3.close()
    rd = _rdatas([SCENES[1]])[0]
    gr = api.GpuRenderer(rd, max_depth=SCENES[1][5]).upload()
    gr.set_tune(block=128, stack=32, fuse=2)
    want = gr.get_tune()
    gr.tune_save(path)
    gr.close()
    gr2 = api.GpuRenderer(rd, max_depth=SCENES[1][5]).upload()
    assert gr2.tune_load(path) == 1
    got = gr2.get_tune()
    assert all(got[k] == want[k] for k in keys)
    gr2.close()
    assert len(open(path).read().splitlines()) == 2


def test_batched_radiance_cache(gpu):
    """RENDGPU_MODE_NRC in a batch: one cache serves every scene (each in
    its own encoding box, the scenes told apart by input features).  The
    warm-up frame, which traces every path unbiased while the cache trains,
    is bit-identical to each scene's own warm-up frame; later frames end
    paths in the cache of every scene, and its images stay as close to a
    converged reference as each scene's own cache gets."""
    from nodebleed_b200 import nrc_eval
    scenes = SCENES[1:3]
    depths = [s[5] for s in scenes]
    rds = _rdatas(scenes)
    b = api.BatchRenderer(rds, max_depth=depths, mode=api.MODE_NRC,
                          seed=7).upload()
    b.frame()
    b.readback(1)
    warm = [rd.acc().copy() for rd in rds]
    tot, _ = b.stats()
    assert tot["nrc_records"] > 0 and tot["nrc_queries"] == 0
    frames = 6
    for _ in range(frames - 1):
        b.frame()
        tot, per = b.stats()
        assert tot["nrc_queries"] > 0 and tot["device_errors"] == 0
    b.readback(1)
    got = [rd.acc() / rd.rd.samples for rd in rds]
    b.close()

    def relmse(x, r):
        return float(np.mean((x - r) ** 2 / (r ** 2 + 1e-2)))
    for i, (fam, seed, w, h, spp, depth) in enumerate(scenes):
        rd = _rdatas([scenes[i]])[0]
        g = api.GpuRenderer(rd, max_depth=depth, mode=api.MODE_NRC,
                            seed=7).upload()
        g.frame()
        g.readback(1)
        assert np.array_equal(rd.acc(), warm[i]), i
        for _ in range(frames - 1):
            g.frame()
        g.readback(1)
        alone = rd.acc() / rd.rd.samples
        g.close()
        ref = nrc_eval.reference(api.Scene(fam, seed), w, h, depth, 256)
        e_b, e_a = relmse(got[i], ref), relmse(alone, ref)
        print(f"scene {i}: relMSE batched cache {e_b:.4f}, own cache "
              f"{e_a:.4f}")
        assert np.isfinite(got[i]).all()
        # measured 0.0006 / 0.0006 and 0.0028 / 0.0027; the order of the
        # device-side record appends varies from run to run
        assert e_b <= 1.5 * e_a + 5e-4, (i, e_b, e_a)


@pytest.mark.parametrize("tune", [{"sort": 1}, {"sort": 1, "queue": 9000}])
def test_ray_reordering_changes_no_bits(gpu, tune):
    """Reordering each bounce's rays (single-scene contexts) leaves every
    path's result unchanged."""
    scenes = [SCENES[1]]
    base, rays0 = _alone(frames=2, scenes=scenes)
    rd = _rdatas(scenes)[0]
    gr = api.GpuRenderer(rd, max_depth=scenes[0][5], seed=7).upload()
    gr.set_tune(**tune)
    assert gr.get_tune()["sort"] == 1
    rays = []
    for _ in range(2):
        gr.frame()
        st = gr.stats()
        rays.append((st["closest_rays"], st["shadow_rays"]))
    gr.readback(1)
    assert np.array_equal(rd.acc(), base[0])
    assert rays == rays0[0]
    gr.close()
