"""Batched compress (gpz_batch_*): every snapshot of a mixed batch gives the
same stream bytes and results as a single gpz_compress call with the same
parameters, launch after launch of the same plan.  CPU tests cover the
descriptor layout and the argument checks that run before any CUDA call."""
import ctypes

import numpy as np
import pytest

import gpz_b200 as gz


def test_batch_item_layout_matches_the_header():
    assert ctypes.sizeof(gz.BatchItem) == 88
    assert gz.BatchItem.flags.offset == 80 and gz.BatchItem.eb.offset == 56


@pytest.mark.parametrize("field,value", [("float_bits", 16), ("dim", 4), ("n", 0), ("d_out", None),
                                         ("flags", 8), ("out_capacity", 10)])
def test_batch_create_rejects_bad_items_before_touching_the_gpu(field, value):
    good = dict(float_bits=32, dim=3, n=5000, d_x=0x1000, d_y=0x2000, d_z=0x3000, d_out=0x4000,
                out_capacity=1 << 20, eb=0.1, rel_eb=0.0, rel_mode=0, seg_size=0, flags=0, reserved=0)
    items = (gz.BatchItem * 3)(gz.BatchItem(**good), gz.BatchItem(**good), gz.BatchItem(**dict(good, **{field: value})))
    h, bad = ctypes.c_void_p(), ctypes.c_uint32(99)
    assert gz.lib().gpz_batch_create(items, 3, ctypes.byref(h), ctypes.byref(bad)) == gz.GPZ_EINVAL
    assert bad.value == 2 and not h.value


def test_batch_create_rejects_fixed_segment_zero():
    it = gz.BatchItem(float_bits=64, dim=2, n=10, d_x=1, d_y=1, d_z=None, d_out=1, out_capacity=1 << 16, eb=1.0,
                      rel_eb=0.0, rel_mode=0, seg_size=0, flags=gz.GPZ_FLAG_SEG_FIXED, reserved=0)
    h, bad = ctypes.c_void_p(), ctypes.c_uint32(99)
    assert gz.lib().gpz_batch_create((gz.BatchItem * 1)(it), 1, ctypes.byref(h), ctypes.byref(bad)) == gz.GPZ_EINVAL
    assert bad.value == 0


# ---------------------------------------------------------------------------- GPU

def _mixed_snapshots():
    """(x, y, z, params) for a batch covering both float widths, 2D/3D,
    device rel bounds, given bounds, fixed / automatic / given segment
    sizes, ragged and single-chunk sizes, and the SAFE31 rules."""
    import torch
    from oracle import pyoracle as po
    cases = [
        # kind, n, dim, bits, kwargs
        (0, 1, 3, 32, dict(eb=0.5, rel_mode=False, seg_size=4)),
        (1, 1000, 3, 32, dict(rel_eb=1e-4)),
        (1, 1025, 2, 32, dict(eb=0.25, rel_mode=False, seg_size=8)),
        (0, 50_003, 3, 32, dict(rel_eb=1e-5)),
        (1, 300_000, 3, 32, dict(rel_eb=1e-4)),
        (2, 70_000, 2, 64, dict(rel_eb=1e-5)),
        (1, 123_456, 3, 64, dict(eb=0.05, rel_mode=False, seg_size=16, fixed=True)),
        (0, 8192, 2, 32, dict(rel_eb=1e-3, seg_size=4)),
        (2, 40_000, 3, 64, dict(rel_eb=1e-5, safe31=True)),
        (1, 262_144, 3, 32, dict(eb=0.1, rel_eb=1e-4, rel_mode=True)),
        (0, 2047, 3, 64, dict(rel_eb=1e-3)),
        (1, 99_999, 2, 32, dict(rel_eb=1e-4)),
    ]
    out = []
    for i, (kind, n, dim, bits, kw) in enumerate(cases):
        dt = np.float32 if bits == 32 else np.float64
        x, y, z = (torch.from_numpy(a.copy()).cuda() for a in po.generate(kind, n, dim, 0.0, 300.0 + 50 * i, 40 + i, dt))
        out.append((x, y, z if dim == 3 else None, kw))
    return out


def _single(x, y, z, kw, bits):
    """The same snapshot through gz.compress (one call)."""
    rel = kw.get("rel_eb", 0.0)
    if kw.get("eb") is None:
        eb, _ = gz.rel_to_abs(x, y, z, rel)
        rel_mode = True
    else:
        eb, rel_mode = kw["eb"], kw.get("rel_mode", False)
    p = gz.make_params(x.numel(), 3 if z is not None else 2, bits, eb, kw.get("seg_size", 0), rel_mode, rel,
                       kw.get("safe31", False))
    if kw.get("fixed"):
        p.flags |= gz.GPZ_FLAG_SEG_FIXED
    import torch
    out = torch.empty(gz.stream_bound(x.numel(), p.dim, bits), dtype=torch.uint8, device=x.device)
    scratch = torch.empty(gz.compress_scratch_bytes(x.numel()), dtype=torch.uint8, device=x.device)
    r = gz.compress_into(p, x, y, z if z is not None else x, out, scratch)
    return out[: r.stream_bytes].cpu().numpy().tobytes(), r, float((np.float32 if bits == 32 else np.float64)(eb))


@pytest.mark.gpu
def test_batch_streams_equal_single_calls():
    from gpz_b200.batch import Batch, Snapshot
    snaps = _mixed_snapshots()
    b = Batch([Snapshot(x, y, z, **kw) for x, y, z, kw in snaps])
    try:
        for launch in range(2):  # the plan's graph replays to the same bytes
            for s in b.snapshots:
                s.out.fill_(0xAB)
            b.launch()
            res = b.results()
            for i, ((x, y, z, kw), s, (r, eb)) in enumerate(zip(snaps, b.snapshots, res)):
                bits = 32 if x.dtype.itemsize == 4 else 64
                want, r1, eb1 = _single(x, y, z, kw, bits)
                assert r.status == 0, (i, r.status)
                assert eb == eb1, (i, eb, eb1)
                assert (r.seg_size, r.adjusted, r.id_overflow) == (r1.seg_size, r1.adjusted, r1.id_overflow), i
                assert r.stream_bytes == r1.stream_bytes, (i, r.stream_bytes, r1.stream_bytes)
                assert s.out[: r.stream_bytes].cpu().numpy().tobytes() == want, (launch, i)
    finally:
        b.close()


@pytest.mark.gpu
def test_batch_reports_a_failed_snapshot_and_finishes_the_others():
    """abs mode without a segment size has no automatic choice (GPZ_EINVAL on
    the single call); in a batch that snapshot reports its status and the
    others are unaffected."""
    import torch
    from gpz_b200.batch import Batch, Snapshot
    from oracle import pyoracle as po
    x, y, z = (torch.from_numpy(a.copy()).cuda() for a in po.generate(1, 30_000, 3, 0.0, 100.0, 3, np.float32))
    b = Batch([Snapshot(x, y, z, rel_eb=1e-4), Snapshot(x, y, z, eb=0.1, rel_mode=False, seg_size=0),
               Snapshot(x, y, z, eb=0.1, rel_mode=False, seg_size=8)])
    try:
        b.launch()
        res = b.results()
        assert res[0][0].status == 0 and res[2][0].status == 0
        assert res[1][0].status != 0
        want, _, _ = _single(x, y, z, dict(eb=0.1, rel_mode=False, seg_size=8), 32)
        assert b.snapshots[2].out[: res[2][0].stream_bytes].cpu().numpy().tobytes() == want
    finally:
        b.close()


@pytest.mark.gpu
def test_decompress_batch_equals_single_calls():
    """The batch's streams decoded by one DecompressBatch launch equal
    gz.decompress of each stream, bit for bit, on two launches; a corrupted
    stream in the batch reports GPZ_ESTREAM without disturbing the others."""
    import torch
    from gpz_b200.batch import Batch, DecompressBatch, Snapshot
    snaps = _mixed_snapshots()
    b = Batch([Snapshot(x, y, z, **kw) for x, y, z, kw in snaps])
    try:
        b.launch()
        streams = [t.clone() for t in b.streams()]
    finally:
        b.close()
    bad = streams[4].clone()
    hb = 24
    G = (snaps[4][0].numel() + 1023) // 1024
    bad[hb + 8 * G + 36 * 1 + 34] = 0xFF  # chunk 1's U field: impossible
    bad[hb + 8 * G + 36 * 1 + 35] = 0xFF
    d = DecompressBatch(streams + [bad])
    try:
        for _ in range(2):
            for o in d.outputs:
                for t in o:
                    if t is not None:
                        t.fill_(-1.0)
            d.launch()
            st = d.results()
            assert st[:-1] == [0] * len(streams) and st[-1] == gz.GPZ_ESTREAM
            for s, o in zip(streams, d.outputs):
                want = gz.decompress(s)
                for a, w in zip(o, want):
                    if w is None:
                        assert a is None
                    else:
                        assert torch.equal(a.view(torch.uint8), w.view(torch.uint8))
    finally:
        d.close()


@pytest.mark.gpu
def test_autotune_picks_the_smallest_sample_and_keeps_bytes_identical():
    """The tuner's choice is the candidate with the smallest sample stream;
    the batch compressed with the tuned segment sizes equals single calls with
    the same fixed segment sizes."""
    from gpz_b200.batch import Batch, Snapshot, autotune
    snaps = _mixed_snapshots()[1:6]
    snapshots = [Snapshot(x, y, z, **kw) for x, y, z, kw in snaps]
    recs = autotune(snapshots, sample_points=20_000)
    for s, rec, (x, y, z, kw) in zip(snapshots, recs, snaps):
        if kw.get("seg_size") or kw.get("fixed"):
            assert rec == {}
            continue
        assert rec["sample_bytes"] and s.fixed and s.seg_size == rec["seg"]
        assert rec["sample_bytes"][rec["seg"]] == min(rec["sample_bytes"].values())
    b = Batch(snapshots)
    try:
        b.launch()
        res = b.results()
        for s, (r, eb), (x, y, z, kw) in zip(snapshots, res, snaps):
            bits = 32 if x.dtype.itemsize == 4 else 64
            kw2 = dict(kw, seg_size=s.seg_size, fixed=True)
            want, r1, eb1 = _single(x, y, z, kw2, bits)
            assert r.status == 0 and eb == eb1 and r.seg_size == s.seg_size
            assert s.out[: r.stream_bytes].cpu().numpy().tobytes() == want
    finally:
        b.close()
