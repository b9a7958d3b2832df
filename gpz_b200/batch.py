"""Batched compress of many snapshots (gpz_batch_* of the C ABI).

A `Batch` is a plan bound to its snapshots' device buffers: it is created
once (validation, device memory for descriptors and per-snapshot control
blocks, CUDA-graph capture) and launched any number of times; each launch
compresses every snapshot, and each snapshot's stream is byte-identical to
what `gpz_b200.compress` writes with the same parameters.  The reference has
no batched form (one snapshot per CompressorManager::compressWarp call,
reference src/CompressorManager.cpp:12-16).

    snaps = [Snapshot(x, y, z, rel_eb=1e-4), Snapshot(x2, y2, None, eb=0.5, seg_size=8)]
    b = Batch(snaps)
    b.launch()
    streams = b.streams()          # uint8 CUDA tensors, one per snapshot
    b.close()

`DecompressBatch` is the reverse: many streams decoded by one graph launch.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

from . import (BatchItem, DBatchItem, GPZ_FLAG_REL_ON_DEVICE, GPZ_FLAG_SAFE31, GPZ_FLAG_SEG_FIXED, GpzError, Result,
               _check, _dtype_bits, _stream_ptr, lib, parse_header, stream_bound)


@dataclass
class Snapshot:
    """One snapshot: SoA CUDA tensors (z None for 2D) and its bound.

    rel_eb given and eb None: the absolute bound is computed on the device
    (as gpz_rel_to_abs does) and the segment-size rules run in "rel" mode.
    eb given: that absolute bound; rel_mode / rel_eb only steer the
    automatic segment size.  seg_size 0 = automatic; fixed=True uses
    seg_size as is (no sampling)."""
    x: object
    y: object
    z: object = None
    eb: float | None = None
    rel_eb: float = 0.0
    rel_mode: bool | None = None
    seg_size: int = 0
    fixed: bool = False
    safe31: bool = False
    out: object = field(default=None, repr=False)

    def item(self) -> BatchItem:
        torch = __import__("torch")
        dim = 3 if self.z is not None else 2
        bits = _dtype_bits(self.x)
        n = self.x.numel()
        if self.out is None:
            self.out = torch.empty(stream_bound(n, dim, bits), dtype=torch.uint8, device=self.x.device)
        flags = (GPZ_FLAG_SEG_FIXED if self.fixed else 0) | (GPZ_FLAG_SAFE31 if self.safe31 else 0)
        rel_mode = self.rel_mode if self.rel_mode is not None else self.eb is None
        if self.eb is None:
            flags |= GPZ_FLAG_REL_ON_DEVICE
        return BatchItem(float_bits=bits, dim=dim, n=n, d_x=self.x.data_ptr(), d_y=self.y.data_ptr(),
                         d_z=self.z.data_ptr() if dim == 3 else None, d_out=self.out.data_ptr(),
                         out_capacity=self.out.numel(), eb=float(self.eb or 0.0), rel_eb=float(self.rel_eb),
                         rel_mode=1 if rel_mode else 0, seg_size=int(self.seg_size), flags=flags, reserved=0)


class Batch:
    def __init__(self, snapshots: list[Snapshot]):
        self.snapshots = list(snapshots)
        n = len(self.snapshots)
        self._items = (BatchItem * n)(*[s.item() for s in self.snapshots])
        self._h = ctypes.c_void_p()
        bad = ctypes.c_uint32(0)
        rc = lib().gpz_batch_create(self._items, n, ctypes.byref(self._h), ctypes.byref(bad))
        if rc:
            raise GpzError(rc, f"gpz_batch_create (item {bad.value})" if rc == 1 else "gpz_batch_create")
        self._results = None

    @property
    def device_bytes(self) -> int:
        return int(lib().gpz_batch_device_bytes(self._h))

    def launch(self, stream=None) -> None:
        """Enqueues one compress of every snapshot (a CUDA graph launch)."""
        self._results = None
        _check(lib().gpz_batch_launch(self._h, _stream_ptr(stream)), "gpz_batch_launch")

    def results(self, stream=None) -> list[tuple[Result, float]]:
        """Synchronises `stream`; (Result, absolute bound) per snapshot."""
        n = len(self.snapshots)
        res = (Result * n)()
        ebs = (ctypes.c_double * n)()
        _check(lib().gpz_batch_results(self._h, res, ebs, _stream_ptr(stream)), "gpz_batch_results")
        self._results = [(res[i], ebs[i]) for i in range(n)]
        return self._results

    def streams(self, stream=None):
        """Each snapshot's stream as a uint8 CUDA tensor view (raises on a failed snapshot)."""
        out = []
        for s, (r, _) in zip(self.snapshots, self._results or self.results(stream)):
            if r.status:
                raise GpzError(r.status, "batched compress")
            out.append(s.out[: r.stream_bytes])
        return out

    def close(self) -> None:
        if self._h:
            lib().gpz_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DecompressBatch:
    """Decodes many streams (uint8 CUDA tensors) with one graph launch; the
    outputs are allocated here (SoA, one tensor per axis, None for z in 2D)."""

    def __init__(self, streams: list):
        torch = __import__("torch")
        self.streams = list(streams)
        self.outputs = []
        items = []
        for st in self.streams:
            h = parse_header(st[:32].cpu().numpy().tobytes())
            dt = torch.float32 if h["float_bits"] == 32 else torch.float64
            n, dim = h["n"], h["dim"]
            xyz = [torch.empty(n, dtype=dt, device=st.device) for _ in range(dim)]
            self.outputs.append((xyz[0], xyz[1], xyz[2] if dim == 3 else None))
            items.append(DBatchItem(d_stream=st.data_ptr(), stream_bytes=st.numel(), float_bits=h["float_bits"], dim=dim,
                                    n=n, d_x=xyz[0].data_ptr(), d_y=xyz[1].data_ptr(),
                                    d_z=xyz[2].data_ptr() if dim == 3 else None, out_capacity=n))
        self._items = (DBatchItem * len(items))(*items)
        self._h = ctypes.c_void_p()
        bad = ctypes.c_uint32(0)
        rc = lib().gpz_dbatch_create(self._items, len(items), ctypes.byref(self._h), ctypes.byref(bad))
        if rc:
            raise GpzError(rc, f"gpz_dbatch_create (item {bad.value})" if rc == 1 else "gpz_dbatch_create")

    def launch(self, stream=None) -> None:
        _check(lib().gpz_dbatch_launch(self._h, _stream_ptr(stream)), "gpz_dbatch_launch")

    def results(self, stream=None) -> list[int]:
        """Synchronises `stream`; the status of every stream."""
        n = len(self.streams)
        res = (Result * n)()
        _check(lib().gpz_dbatch_results(self._h, res, _stream_ptr(stream)), "gpz_dbatch_results")
        return [res[i].status for i in range(n)]

    def close(self) -> None:
        if self._h:
            lib().gpz_dbatch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _block_ids_fit(mm6, dim: int, seg: int, eb: float) -> bool:
    """True when block_num^dim stays below 2^31 for the whole snapshot's range
    (then no chunk's block ids can reach the reference's 31-bit mask)."""
    import math
    if eb <= 0:
        return False
    tot = 1
    for d in range(dim):
        rng = mm6[3 + d] - mm6[d]
        tot *= math.ceil(rng / (2.0 * seg * eb)) + 1
    return tot < (1 << 31)


def autotune(snapshots: list[Snapshot], candidates=(1, 2, 4, 8, 16, 32, 64, 128), sample_points: int = 1 << 17,
             stream=None) -> list[dict]:
    """Picks each snapshot's segment size by compressed size.

    For every snapshot whose segment size is automatic, the first
    `sample_points` points are compressed once per candidate segment size
    (powers of two whose block ids fit in 31 bits over the snapshot's whole
    range) -- all samples of all snapshots in one batched launch -- and the
    candidate with the smallest stream wins; ties go to the larger segment.
    The snapshot is then set to that fixed segment size (its bound keeps its
    mode: a device rel->abs bound stays one).  Returns, per snapshot, the
    record {"seg", "eb", "sample_points", "sample_bytes": {seg: bytes}} (an
    empty dict for snapshots whose segment size was given)."""
    from . import rel_to_abs
    jobs, owners, records = [], [], []
    for i, s in enumerate(snapshots):
        if s.fixed or s.seg_size:
            records.append({})
            continue
        rel = s.rel_eb
        eb_dev, mm = rel_to_abs(s.x, s.y, s.z, rel if s.eb is None else 1.0, stream)
        eb = eb_dev if s.eb is None else float(s.eb)
        dim = 3 if s.z is not None else 2
        m = min(s.x.numel(), sample_points)
        cands = [c for c in candidates if _block_ids_fit(mm, dim, c, eb)]
        records.append({"sample_points": m, "sample_bytes": {}, "eb": eb})
        for c in cands:
            jobs.append(Snapshot(s.x[:m], s.y[:m], s.z[:m] if s.z is not None else None, eb=eb, rel_eb=rel,
                                 rel_mode=True, seg_size=c, fixed=True))
            owners.append((i, c))
    if jobs:
        b = Batch(jobs)
        try:
            b.launch(stream)
            res = b.results(stream)
        finally:
            b.close()
        for (i, c), (r, _) in zip(owners, res):
            if r.status == 0:
                records[i]["sample_bytes"][c] = int(r.stream_bytes)
    for i, s in enumerate(snapshots):
        rec = records[i]
        if not rec or not rec["sample_bytes"]:
            continue
        best = min(rec["sample_bytes"].items(), key=lambda kv: (kv[1], -kv[0]))[0]
        rec["seg"] = best
        s.seg_size, s.fixed = best, True
    return records
