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
