"""Request server (gpz_server_* of the C ABI): continuous batching of compress
and decompress requests under a device-memory budget.

    srv = Server(hbm_budget=8 << 30, streams=3, max_batch=64)
    t = srv.submit_compress(x, y, z, rel_eb=1e-4)      # returns at once
    c = srv.wait(t)                                     # Completion
    stream = srv.stream_view(t, c)                      # uint8 CUDA tensor (a view into the arena)
    srv.release(t)                                      # the output's memory goes back to the budget

Outputs live in the server's arena until released; views of them must not be
used after release.  The reference has no serving form (it is a command line
tool that compresses one file per run).
"""
from __future__ import annotations

import ctypes
import threading

from . import (Completion, GPZ_FLAG_REL_ON_DEVICE, GPZ_FLAG_SAFE31, GPZ_FLAG_SEG_FIXED, GPZ_OP_COMPRESS,
               GPZ_OP_DECOMPRESS, GPZ_SERVER_OVERLAP, GpzError, Request, ServerConfig, ServerStats, _check,
               _dtype_bits, lib, parse_header)


class _DeviceBuffer:
    """A raw device range exposed through __cuda_array_interface__."""

    def __init__(self, ptr: int, shape: tuple, typestr: str):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (ptr, False), "version": 3,
                                         "strides": None}


class Server:
    def __init__(self, hbm_budget: int, streams: int = 3, max_batch: int = 64, workspace_bytes: int = 0,
                 overlap: bool = False):
        cfg = ServerConfig(hbm_budget=hbm_budget, streams=streams, max_batch=max_batch,
                           workspace_bytes=workspace_bytes, flags=GPZ_SERVER_OVERLAP if overlap else 0, reserved=0)
        self._h = ctypes.c_void_p()
        _check(lib().gpz_server_create(ctypes.byref(cfg), ctypes.byref(self._h)), "gpz_server_create")
        self._keep = {}  # ticket -> (inputs kept alive until completion, output description)
        self._lock = threading.Lock()

    def _submit(self, req: Request, keep) -> int:
        t = ctypes.c_uint64()
        _check(lib().gpz_server_submit(self._h, ctypes.byref(req), ctypes.byref(t)), "gpz_server_submit")
        with self._lock:
            self._keep[t.value] = keep
        return t.value

    def submit_compress(self, x, y, z=None, eb: float | None = None, rel_eb: float = 0.0, rel_mode: bool | None = None,
                        seg_size: int = 0, fixed: bool = False, safe31: bool = False) -> int:
        """Compress SoA CUDA tensors; eb None = absolute bound computed on the
        device from rel_eb (as gpz_rel_to_abs)."""
        dim = 3 if z is not None else 2
        flags = (GPZ_FLAG_SEG_FIXED if fixed else 0) | (GPZ_FLAG_SAFE31 if safe31 else 0)
        if eb is None:
            flags |= GPZ_FLAG_REL_ON_DEVICE
        rm = rel_mode if rel_mode is not None else eb is None
        req = Request(op=GPZ_OP_COMPRESS, float_bits=_dtype_bits(x), dim=dim, flags=flags, n=x.numel(),
                      d_x=x.data_ptr(), d_y=y.data_ptr(), d_z=z.data_ptr() if dim == 3 else None, d_stream=None,
                      stream_bytes=0, eb=float(eb or 0.0), rel_eb=float(rel_eb), rel_mode=1 if rm else 0,
                      seg_size=int(seg_size))
        return self._submit(req, ((x, y, z), None))

    def submit_decompress(self, stream, header: dict | None = None) -> int:
        """Decompress a stream held in a uint8 CUDA tensor."""
        h = header or parse_header(stream[:32].cpu().numpy().tobytes())
        req = Request(op=GPZ_OP_DECOMPRESS, float_bits=h["float_bits"], dim=h["dim"], flags=0, n=h["n"], d_x=None,
                      d_y=None, d_z=None, d_stream=stream.data_ptr(), stream_bytes=stream.numel(), eb=0.0,
                      rel_eb=0.0, rel_mode=0, seg_size=0)
        return self._submit(req, ((stream,), h))

    def wait(self, ticket: int, timeout_ms: int = 0) -> Completion:
        c = Completion()
        _check(lib().gpz_server_wait(self._h, ticket, ctypes.byref(c), timeout_ms), "gpz_server_wait")
        return c

    def stream_view(self, ticket: int, c: Completion):
        """The compressed stream of a completed compress request (a view)."""
        import torch
        if c.status:
            raise GpzError(c.status, "served compress")
        return torch.as_tensor(_DeviceBuffer(c.d_out, (int(c.stream_bytes),), "|u1"), device="cuda")

    def arrays_view(self, ticket: int, c: Completion):
        """(x, y, z) of a completed decompress request (views; z None in 2D)."""
        import torch
        if c.status:
            raise GpzError(c.status, "served decompress")
        h = self._keep[ticket][1]
        n, dim, bits = h["n"], h["dim"], h["float_bits"]
        stride = (n * bits // 8 + 255) & ~255
        ts = "<f4" if bits == 32 else "<f8"
        out = [torch.as_tensor(_DeviceBuffer(c.d_out + k * stride, (n,), ts), device="cuda") for k in range(dim)]
        return out[0], out[1], out[2] if dim == 3 else None

    def release(self, ticket: int) -> None:
        _check(lib().gpz_server_release(self._h, ticket), "gpz_server_release")
        with self._lock:
            self._keep.pop(ticket, None)

    def stats(self) -> ServerStats:
        st = ServerStats()
        _check(lib().gpz_server_stats_get(self._h, ctypes.byref(st)), "gpz_server_stats_get")
        return st

    def close(self) -> None:
        if self._h:
            lib().gpz_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
