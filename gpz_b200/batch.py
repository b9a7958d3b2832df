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
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

from . import (BatchItem, GPZ_FLAG_REL_ON_DEVICE, GPZ_FLAG_SAFE31, GPZ_FLAG_SEG_FIXED, GpzError, Result, _check,
               _dtype_bits, _stream_ptr, lib, stream_bound)


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
