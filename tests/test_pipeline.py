"""Host-memory round trips with overlapped copies (gpz_b200.pipeline): the
stream and reconstruction of every step equal the single-call ones."""
import numpy as np
import pytest

import gpz_b200 as gz
from gpz_b200.pipeline import SnapshotPipeline


def test_rejects_bad_shapes_before_allocating():
    for dim, bits in ((4, 32), (3, 16), (1, 64)):
        with pytest.raises(gz.GpzError):
            SnapshotPipeline(gz.make_params(1000, 3, 32, 0.1), 1000, dim, bits)


@pytest.mark.gpu
@pytest.mark.parametrize("n,dim,bits,steps,abs_eb", [(300_000, 3, 32, 3, 0.0), (70_001, 2, 64, 4, 0.0),
                                                     (50_000, 3, 64, 1, 0.0), (1, 3, 32, 2, 0.01)])
def test_round_trips_equal_single_calls(n, dim, bits, steps, abs_eb):
    import torch
    from oracle import pyoracle as po
    dt = np.float32 if bits == 32 else np.float64
    x, y, z = po.generate(1, n, dim, 0.0, 500.0, 31, dt)
    dev = [torch.from_numpy(a.copy()).cuda() for a in (x, y, z)]
    zz = dev[2] if dim == 3 else None
    if abs_eb:  # one point has no range for a relative bound
        eb, rel, seg = abs_eb, 0.0, 4
    else:
        (eb, _), rel, seg = gz.rel_to_abs(dev[0], dev[1], zz, 1e-4), float(dt(1e-4)), 0
    want, r = gz.compress(dev[0], dev[1], zz, eb=eb, seg_size=seg, rel_mode=not abs_eb, rel_eb=rel)
    wx, wy, wz = gz.decompress(want)
    host = [torch.from_numpy(a.copy()).pin_memory() for a in (x, y, z)][:dim]
    p = gz.make_params(n, dim, bits, eb, seg, not abs_eb, rel)
    pipe = SnapshotPipeline(p, n, dim, bits)
    nb, rx = pipe.round_trips(host, steps)
    assert nb == r.stream_bytes
    for k in range(2):
        if pipe.nb[k]:
            assert torch.equal(pipe.hs[k][:nb].cuda(), want)
    for h, w in zip(rx, (wx, wy, wz)):
        assert torch.equal(h.view(torch.uint8), w.cpu().view(torch.uint8))


@pytest.mark.gpu
def test_result_post_matches_result_get_and_rejects_pageable_memory():
    import ctypes
    import torch
    n = 50_000
    x, y, z = (torch.rand(n, device="cuda") * 100 for _ in range(3))
    p = gz.make_params(n, 3, 32, 0.01, 8)
    out = torch.empty(gz.stream_bound(n, 3, 32), dtype=torch.uint8, device="cuda")
    scr = torch.empty(gz.compress_scratch_bytes(n), dtype=torch.uint8, device="cuda")
    want = gz.compress_into(p, x, y, z, out, scr)
    host = torch.zeros(64, dtype=torch.uint8).pin_memory()
    gz.result_post(scr, host)
    torch.cuda.synchronize()
    got = gz.Result.from_buffer_copy(host.numpy().tobytes()[:ctypes.sizeof(gz.Result)])
    assert (got.stream_bytes, got.seg_size, got.status) == (want.stream_bytes, want.seg_size, want.status)
    pageable = (ctypes.c_uint8 * 64)()
    assert gz.lib().gpz_result_post(scr.data_ptr(), ctypes.addressof(pageable), None) == gz.GPZ_EINVAL
    with pytest.raises(gz.GpzError):
        gz.result_post(scr, torch.zeros(64, dtype=torch.uint8))


STAGES = ["upload", "compress", "stream_size", "download_stream", "upload_stream", "decompress", "fetch"]


@pytest.mark.parametrize("steps", [1, 2, 3, 4, 7])
def test_schedule_orders_stages_and_slot_reuse(steps):
    """The host schedule, stages stubbed: each step's stages in dependency
    order, each once, and a slot refilled only after the previous step on
    that slot has issued the stage that reads it (the event every wait names
    must already be recorded when the wait is enqueued)."""
    pipe = object.__new__(SnapshotPipeline)
    log = []
    for name in STAGES:
        setattr(pipe, name, (lambda nm: lambda k, *a: log.append((nm, k)))(name))
    pipe.synchronize = lambda: log.append(("sync", -1))
    pipe.nb, pipe.rX = [0, 0], [[], []]
    pipe.round_trips([None], steps)
    assert log[-1] == ("sync", -1)
    seen, pos = {}, {}
    for idx, (nm, k) in enumerate(log[:-1]):
        j = seen.get((nm, k), 0)
        seen[(nm, k)] = j + 1
        pos[(nm, 2 * j + k)] = idx  # the j-th use of slot k is step 2j + k
    assert sorted(pos) == sorted((nm, i) for nm in STAGES for i in range(steps))
    for i in range(steps):
        for a, b in zip(STAGES, STAGES[1:]):
            assert pos[(a, i)] < pos[(b, i)], (i, a, b)
    for i in range(2, steps):
        assert pos[("compress", i - 2)] < pos[("upload", i)]
        assert pos[("download_stream", i - 2)] < pos[("compress", i)]
        assert pos[("upload_stream", i - 2)] < pos[("download_stream", i)]
        assert pos[("decompress", i - 2)] < pos[("upload_stream", i)]
        assert pos[("fetch", i - 2)] < pos[("decompress", i)]


def test_schedule_rejects_zero_steps():
    pipe = object.__new__(SnapshotPipeline)
    with pytest.raises(gz.GpzError):
        pipe.round_trips([None], 0)
