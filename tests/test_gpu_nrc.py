"""Neural radiance cache kernels on the GPU (rendgpu_nrc_*) against the FP64
oracle (oracle/nrc_oracle.py): encoding, forward pass, gradients, Adam."""

import ctypes as C
import os
import sys

import numpy as np
import pytest

from nodebleed_b200 import api

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(
    os.path.abspath(__file__))), "oracle"))
import nrc_oracle as no  # noqa: E402

pytestmark = pytest.mark.gpu


def _setup(seed=7):
    """Renderer with Xavier-initialised weights in every layer (the
    library starts the output layer at zero)."""
    scene = api.Scene(api.SCENE_TINY, 1)
    rd = api.RenderData(scene)
    gr = api.GpuRenderer(rd).upload()
    gr.nrc_reset(seed)
    gr.nrc_weights(no.xavier(seed).astype(np.float32))
    return rd, gr


def _box(rd):
    r = rd.rd
    a = np.ctypeslib.as_array((C.c_float * (8 * r.instcnt)).from_address(
        r.aabbs)).reshape(-1, 8)
    return a[:, 0:3].min(0).astype(np.float64), \
        a[:, 4:7].max(0).astype(np.float64)


def _dev(x, dtype=None):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(x))
    return t.cuda() if dtype is None else t.to(dtype).cuda()


def _feats_dev(f64):
    """BF16 features on the device (torch bfloat16), and their exact
    values as float64."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(f64, np.float32)).to(
        torch.bfloat16).cuda()
    return t, t.float().cpu().numpy().astype(np.float64)


def _random_raw(rd, n, seed=0):
    rng = np.random.default_rng(seed)
    lo, hi = _box(rd)
    raw = np.zeros((n, 12), np.float32)
    raw[:, 0:3] = rng.uniform(lo, hi, (n, 3))
    for s in (3, 6):
        d = rng.normal(size=(n, 3))
        raw[:, s:s + 3] = d / np.linalg.norm(d, axis=1, keepdims=True)
    raw[:, 9:12] = rng.uniform(0, 1, (n, 3))
    return raw


def test_encode_matches_oracle(gpu):
    """All 64 features, the hash grid's with a table of entries in
    [-1, 1] (level 0 and 1 dense, the rest hashed)."""
    import torch
    rd, gr = _setup()
    table = np.random.default_rng(8).uniform(
        -1, 1, no.GRID_PARAMS).astype(np.float32)
    gr.nrc_grid(table)
    assert np.array_equal(gr.nrc_grid(), table)
    raw = _random_raw(rd, 4099)
    out = torch.zeros((len(raw), 64), dtype=torch.bfloat16, device="cuda")
    d_raw = _dev(raw)
    torch.cuda.synchronize()
    gr._ck(gr.g.rendgpu_nrc_encode_device(gr.ptr, d_raw.data_ptr(), len(raw),
                                          out.data_ptr()), "encode")
    gr.g.rendgpu_sync(gr.ptr)
    got = out.float().cpu().numpy()
    lo, hi = _box(rd)
    ref = no.encode(raw, lo.astype(np.float32), hi.astype(np.float32), table)
    err = np.abs(got - ref)
    print(f"encode: max error {err.max():.2e} (grid features "
          f"{err[:, :16].max():.2e})")
    assert err.max() < 8e-3
    assert np.abs(ref[:, :16]).max() > 0.3
    assert (got[:, 48:] == 0).all()
    gr.close()


def _grid_batch(gr, rd, n, seed):
    """A training batch of raw inputs (device) and its targets, with random
    MLP weights and a random table."""
    rng = np.random.default_rng(seed)
    table = rng.uniform(-0.5, 0.5, no.GRID_PARAMS).astype(np.float32)
    gr.nrc_grid(table)
    raw = _random_raw(rd, n, seed)
    t = rng.uniform(0, 2, (n, 4)).astype(np.float32)
    return table, raw, t


@pytest.mark.parametrize("n", [1000, 16384])
def test_grid_gradient_matches_oracle(gpu, n):
    """rendgpu_nrc_train_raw_device: the table's gradient (d loss /
    d feature = dz_0 W_0 spread over the trilinear corners) and the MLP's
    against the oracle on the same BF16-rounded features."""
    import torch
    rd, gr = _setup(13)
    table, raw, t = _grid_batch(gr, rd, n, 5)
    d_raw, d_t = _dev(raw), _dev(t)
    g = torch.zeros(no.NPARAMS, dtype=torch.float32, device="cuda")
    gg = torch.zeros(no.GRID_PARAMS, dtype=torch.float32, device="cuda")
    loss = C.c_float()
    torch.cuda.synchronize()
    gr._ck(gr.g.rendgpu_nrc_train_raw_device(
        gr.ptr, d_raw.data_ptr(), d_t.data_ptr(), n, 0, g.data_ptr(),
        gg.data_ptr(), C.byref(loss)), "train_raw")
    assert gr.g.rendgpu_sync(gr.ptr) == 0
    w = gr.nrc_weights()
    lo, hi = _box(rd)
    lo32, hi32 = lo.astype(np.float32), hi.astype(np.float32)
    feats = no.bf16(no.encode(raw, lo32, hi32, table))
    ref_loss, ref = no.loss_grad(w, feats, t, bf=True)
    dfeat = no.feature_grad(w, feats, t, bf=True)[:, :16]
    x = no.unit_position(raw, lo32, hi32)
    ref_gg = no.grid_grad(x, dfeat)
    got_gg = gg.cpu().numpy().astype(np.float64)
    gerr = np.linalg.norm(got_gg - ref_gg) / np.linalg.norm(ref_gg)
    lerr = abs(loss.value - ref_loss) / ref_loss
    got = g.cpu().numpy().astype(np.float64)
    merr = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    print(f"grid gradient n={n}: relative L2 error {gerr:.3e}, MLP "
          f"{merr:.3e}, loss {lerr:.3e}, entries touched "
          f"{np.count_nonzero(got_gg)}")
    # measured 2.4e-4 (1000 rows) and 1.7e-3 (16384 rows): an entry's
    # gradient comes from the few rows in its cells, so the BF16 rounding
    # of a feature that lands on the other side of a tie (FP32 on the
    # device, FP64 in the oracle) shows in it; the MLP's gradient averages
    # such rows out (4e-5)
    assert gerr < 5e-3
    assert merr < 1e-3
    assert lerr < 1e-4
    # update = 0 leaves the table as it was
    assert np.array_equal(gr.nrc_grid(), table)
    gr.close()


def test_grid_adam_step_matches_oracle(gpu):
    import torch
    rd, gr = _setup(17)
    table, raw, t = _grid_batch(gr, rd, 2048, 6)
    d_raw, d_t = _dev(raw), _dev(t)
    gg = torch.zeros(no.GRID_PARAMS, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    gr._ck(gr.g.rendgpu_nrc_train_raw_device(
        gr.ptr, d_raw.data_ptr(), d_t.data_ptr(), len(raw), 1, None,
        gg.data_ptr(), None), "train_raw")
    assert gr.g.rendgpu_sync(gr.ptr) == 0
    g64 = gg.cpu().numpy().astype(np.float64)
    m = 0.1 * g64
    v = 0.01 * g64 * g64
    ref = table - 1e-2 * (m / 0.1) / (np.sqrt(v / 0.01) + 1e-15)
    got = gr.nrc_grid().astype(np.float64)
    assert np.abs(got - ref).max() < 1e-6
    assert np.count_nonzero(got != table) > 1000
    gr.close()


def test_grid_off_leaves_features_zero(gpu):
    import torch
    scene = api.Scene(api.SCENE_TINY, 1)
    rd = api.RenderData(scene)
    gr = api.GpuRenderer(rd, nrc_grid=False).upload()
    gr.nrc_reset(3)
    raw = _random_raw(rd, 300)
    out = torch.ones((len(raw), 64), dtype=torch.bfloat16, device="cuda")
    d_raw = _dev(raw)
    torch.cuda.synchronize()
    gr._ck(gr.g.rendgpu_nrc_encode_device(gr.ptr, d_raw.data_ptr(), len(raw),
                                          out.data_ptr()), "encode")
    gr.g.rendgpu_sync(gr.ptr)
    got = out.float().cpu().numpy()
    assert (got[:, :16] == 0).all() and (got[:, 16:34] != 0).any()
    gr.close()
    gr.close()


@pytest.mark.parametrize("n", [1, 129, 3001, 200_003])
def test_forward_matches_oracle(gpu, n):
    """Ragged sizes: a single row, one row past a 128-row tile, and a batch
    large enough that every tile pipeline of every CTA runs several tiles
    (and prefetches the next one)."""
    import torch
    rd, gr = _setup()
    rng = np.random.default_rng(1)
    f, f64 = _feats_dev(rng.uniform(0, 1, (n, 64)))
    out = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    gr._ck(gr.g.rendgpu_nrc_infer_device(gr.ptr, f.data_ptr(), n,
                                         out.data_ptr()), "infer")
    gr.g.rendgpu_sync(gr.ptr)
    got = out.cpu().numpy()[:, :3]
    w = gr.nrc_weights()
    _, ref = no.forward(w, f64, bf=True)
    scale = np.abs(ref).max()
    emax = np.abs(got - ref).max() / scale
    emean = np.mean(np.abs(got - ref)) / scale
    print(f"forward n={n}: max error {emax:.3e}, mean error {emean:.3e} "
          "of the output scale")
    # The oracle rounds the same tensors to BF16, so only the order of the
    # FP32 accumulation differs: measured at most 3.6e-3 (a hidden
    # activation whose BF16 rounding flips, carried to the output) and a
    # mean of 7.3e-7 of the output scale.
    assert emax < 8e-3
    assert emean < 1e-5
    gr.close()


def test_query_pass_matches_encode_infer_apply(gpu):
    """rendgpu_nrc_query_device (encode, infer and add to the path's
    radiance in one kernel, as cache frames do) against the separate encode
    and infer calls and the same arithmetic in torch, bit for bit.  150,001
    queries give every tile pipeline several tiles; queries whose path index
    is out of range change nothing."""
    import torch
    rd, gr = _setup(13)
    rng = np.random.default_rng(6)
    n = 150_001
    npath = n + 4000
    raw = _random_raw(rd, n, seed=5)
    paths = rng.permutation(npath)[:n].astype(np.uint32)
    paths[::997] = npath + 3          # skipped
    tput = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    e = np.zeros((n, 4, 4), np.float32)
    for k in range(4):
        e[:, k, :3] = raw[:, 3 * k:3 * k + 3]
    e[:, 0, 3] = paths.view(np.float32)
    e[:, 1:, 3] = tput
    d_e = _dev(e)
    rad = torch.from_numpy(rng.uniform(0, 1, (npath, 4)).astype(
        np.float32)).cuda()
    before = rad.clone()
    d_raw = _dev(raw)
    feats = torch.zeros((n, 64), dtype=torch.bfloat16, device="cuda")
    y = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    gr._ck(gr.g.rendgpu_nrc_query_device(gr.ptr, d_e.data_ptr(), n,
                                         rad.data_ptr(), npath), "query")
    gr._ck(gr.g.rendgpu_nrc_encode_device(gr.ptr, d_raw.data_ptr(), n,
                                          feats.data_ptr()), "encode")
    gr._ck(gr.g.rendgpu_nrc_infer_device(gr.ptr, feats.data_ptr(), n,
                                         y.data_ptr()), "infer")
    assert gr.g.rendgpu_sync(gr.ptr) == 0
    valid = torch.from_numpy(paths < npath).cuda()
    idx = torch.from_numpy(paths.astype(np.int64)).cuda()[valid]
    add = _dev(tput)[valid] * torch.clamp(y[valid, :3], min=0.0)
    want = before.clone()
    want[idx, :3] = before[idx, :3] + add
    assert torch.equal(rad, want)
    assert torch.count_nonzero(add).item() > n // 2
    gr.close()


@pytest.mark.parametrize("cycles", [1_000_000, 20_000_000])
def test_bounded_wait_times_out_and_recovers(gpu, cycles):
    """The tensor-core kernels' waits on their own UMMAs give up after a
    bounded time, so a stuck wait becomes an error status rather than a
    hang.  rendgpu_check_bounded_wait runs that wait on a barrier nothing
    completes (it must time out after its cycle budget, within one poll of
    it), then on one that completes (it must succeed); the context keeps
    working afterwards."""
    import time
    import torch
    rd, gr = _setup()
    out = (C.c_uint32 * 3)()
    t0 = time.perf_counter()
    gr._ck(gr.g.rendgpu_check_bounded_wait(gr.ptr, cycles, out), "check")
    dt = time.perf_counter() - t0
    assert out[0] == 1, "a wait on an unfinished barrier did not time out"
    assert out[1] == 1, "a wait on a finished barrier did not succeed"
    # one try_wait poll suspends the thread for about 8k cycles
    assert cycles <= out[2] < cycles + 200_000, out[2]
    assert dt < 10.0
    f = torch.zeros((256, 64), dtype=torch.bfloat16, device="cuda")
    y = torch.ones((256, 4), dtype=torch.float32, device="cuda")
    gr._ck(gr.g.rendgpu_nrc_infer_device(gr.ptr, f.data_ptr(), 256,
                                         y.data_ptr()), "infer")
    assert gr.g.rendgpu_sync(gr.ptr) == 0
    assert torch.count_nonzero(y[:, :3]).item() == 0
    gr.close()


@pytest.mark.parametrize("n", [2048, 1000, 40_000])
def test_gradients_match_oracle(gpu, n):
    """Per-layer gradients and the loss against the FP64 oracle.  1000 rows
    leave a partial 112-row chunk in the weight-gradient pass; 40,000 rows
    are 313 tiles of 128, so every CTA of the forward/backward pass runs
    several tiles."""
    import torch
    rd, gr = _setup(11)
    rng = np.random.default_rng(2)
    f, f64 = _feats_dev(rng.uniform(0, 1, (n, 64)))
    t = rng.uniform(0, 2, (n, 4)).astype(np.float32)
    d_t = _dev(t)
    g = torch.zeros(no.NPARAMS, dtype=torch.float32, device="cuda")
    loss = C.c_float()
    torch.cuda.synchronize()
    gr._ck(gr.g.rendgpu_nrc_train_device(gr.ptr, f.data_ptr(), d_t.data_ptr(),
                                         n, 0, g.data_ptr(), C.byref(loss)),
           "train")
    gr.g.rendgpu_sync(gr.ptr)
    got = g.cpu().numpy().astype(np.float64)
    w = gr.nrc_weights()
    ref_loss, ref = no.loss_grad(w, f64, t, bf=True)
    # with the oracle rounding the same tensors to BF16 only the FP32
    # accumulation order differs: measured loss error <= 3.4e-7 and
    # per-layer relative L2 errors <= 1.1e-5
    lerr = abs(loss.value - ref_loss) / ref_loss
    assert lerr < 1e-5
    errs = []
    for l in range(6):
        sl = slice(l * no.SQ, (l + 1) * no.SQ) if l < 5 else \
            slice(5 * no.SQ, 5 * no.SQ + 3 * 64)
        err = np.linalg.norm(got[sl] - ref[sl]) / np.linalg.norm(ref[sl])
        errs.append(err)
        assert err < 1e-4, (l, err)
    print(f"gradients n={n}: loss error {lerr:.3e}, per-layer relative L2 "
          "errors " + " ".join(f"{e:.3e}" for e in errs))
    assert (got[5 * no.SQ + 3 * 64:] == 0).all()
    # the weights did not move (update = 0)
    assert np.array_equal(gr.nrc_weights(), w)
    gr.close()


def test_reset_starts_output_layer_at_zero(gpu):
    scene = api.Scene(api.SCENE_TINY, 1)
    rd = api.RenderData(scene)
    gr = api.GpuRenderer(rd).upload()
    gr.nrc_reset(5)
    w = gr.nrc_weights()
    assert (w[5 * no.SQ:] == 0).all()
    assert np.abs(w[:5 * no.SQ]).max() > 0.1
    gr.close()


def test_adam_step_matches_oracle(gpu):
    import torch
    rd, gr = _setup(3)
    w0 = no.xavier(5).astype(np.float32)
    gr.nrc_weights(w0)
    rng = np.random.default_rng(3)
    n = 1024
    f, f64 = _feats_dev(rng.uniform(0, 1, (n, 64)))
    d_t = _dev(rng.uniform(0, 2, (n, 4)).astype(np.float32))
    g = torch.zeros(no.NPARAMS, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    gr._ck(gr.g.rendgpu_nrc_train_device(gr.ptr, f.data_ptr(), d_t.data_ptr(),
                                         n, 1, g.data_ptr(), None), "train")
    gr.g.rendgpu_sync(gr.ptr)
    w1 = gr.nrc_weights().astype(np.float64)
    gg = g.cpu().numpy().astype(np.float64)
    ref, _, _ = no.adam(w0.astype(np.float64), np.zeros(no.NPARAMS),
                        np.zeros(no.NPARAMS), gg, 1)
    assert np.abs(w1 - ref).max() < 1e-6
    gr.close()


def test_training_fits_a_smooth_target(gpu):
    import torch
    rd, gr = _setup(21)
    rng = np.random.default_rng(4)
    n = 8192
    x = rng.uniform(0, 1, (n, 64))
    x[:, 50:] = 0
    f, f64 = _feats_dev(x)
    tgt = np.stack([0.5 + 0.4 * np.sin(3 * f64[:, 0] + f64[:, 1]),
                    0.5 + 0.4 * np.cos(2 * f64[:, 2] - f64[:, 3]),
                    0.3 + 0.2 * f64[:, 4] * f64[:, 5],
                    np.zeros(n)], 1).astype(np.float32)
    d_t = _dev(tgt)
    losses = []
    torch.cuda.synchronize()
    for step in range(300):
        lv = C.c_float()
        gr._ck(gr.g.rendgpu_nrc_train_device(
            gr.ptr, f.data_ptr(), d_t.data_ptr(), n, 1, None,
            C.byref(lv) if step % 50 == 0 or step == 299 else None), "train")
        if step % 50 == 0 or step == 299:
            losses.append(lv.value)
    assert losses[-1] < 0.1 * losses[0], losses
    gr.close()
