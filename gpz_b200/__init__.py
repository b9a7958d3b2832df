"""B200-native GPZ particle compressor: Python host binding over the C ABI.

The compute path is the CUDA library ``gpz_b200/libgpz_b200.so`` (built from
``gpz_b200/csrc`` for sm_100a); this module only moves pointers, sizes and
status codes across ``include/gpz_b200.h``.  There is no CPU fallback:
importing the module fails loudly when the library is missing.

The classes at the bottom mirror the reference's plugin interface
(``CudaConfig``, ``ICudaCompressor``, ``CudaWarpCompress``,
``CudaWarpCompressDouble``, ``CompressorManager`` -- reference
include/cudaCompress.cuh:16-40, include/ICudaCompressor.cuh:6-17,
include/CompressorManager.h:9-28) on torch CUDA tensors, with the same
argument meaning: compress overwrites the caller's SoA input buffer with the
stream and mutates the config's segment size.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgpz_b200.so")

GPZ_OK, GPZ_EINVAL, GPZ_ESEG, GPZ_ESTREAM, GPZ_ENOSPACE, GPZ_ECUDA, GPZ_ETIMEOUT, GPZ_ENOTSUP, GPZ_ELIMIT = range(9)
GPZ_FLAG_SAFE31 = 1
GPZ_FLAG_SEG_FIXED = 2
GPZ_FLAG_STRICT_BOUND = 8
GPZ_FLAG_REL_ON_DEVICE = 4
GPZ_OP_COMPRESS, GPZ_OP_DECOMPRESS = 1, 2
GPZ_SERVER_OVERLAP = 1
ERRORS = {1: "EINVAL", 2: "ESEG", 3: "ESTREAM", 4: "ENOSPACE", 5: "ECUDA", 6: "ETIMEOUT", 7: "ENOTSUP", 8: "ELIMIT"}


class GpzError(RuntimeError):
    def __init__(self, code: int, what: str):
        super().__init__(f"{what} failed: GPZ_{ERRORS.get(code, code)}")
        self.code = code


class Params(ctypes.Structure):
    _fields_ = [("float_bits", ctypes.c_uint32), ("dim", ctypes.c_uint32), ("n", ctypes.c_uint64),
                ("eb", ctypes.c_double), ("rel_eb", ctypes.c_double), ("rel_mode", ctypes.c_int32),
                ("seg_size", ctypes.c_uint32), ("flags", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class Result(ctypes.Structure):
    _fields_ = [("stream_bytes", ctypes.c_uint64), ("seg_size", ctypes.c_uint32), ("adjusted", ctypes.c_uint32),
                ("status", ctypes.c_int32), ("id_overflow", ctypes.c_uint32)]


_VP = ctypes.c_void_p
_U64 = ctypes.c_uint64
_U32 = ctypes.c_uint32


class BatchItem(ctypes.Structure):
    """gpz_batch_item: one snapshot of a batched compress."""
    _fields_ = [("float_bits", ctypes.c_uint32), ("dim", ctypes.c_uint32), ("n", ctypes.c_uint64),
                ("d_x", ctypes.c_void_p), ("d_y", ctypes.c_void_p), ("d_z", ctypes.c_void_p),
                ("d_out", ctypes.c_void_p), ("out_capacity", ctypes.c_uint64), ("eb", ctypes.c_double),
                ("rel_eb", ctypes.c_double), ("rel_mode", ctypes.c_int32), ("seg_size", ctypes.c_uint32),
                ("flags", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget", ctypes.c_uint64), ("streams", ctypes.c_uint32), ("max_batch", ctypes.c_uint32),
                ("workspace_bytes", ctypes.c_uint64), ("flags", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class Request(ctypes.Structure):
    """gpz_request: one compress or decompress request to a server."""
    _fields_ = [("op", ctypes.c_uint32), ("float_bits", ctypes.c_uint32), ("dim", ctypes.c_uint32),
                ("flags", ctypes.c_uint32), ("n", ctypes.c_uint64), ("d_x", ctypes.c_void_p),
                ("d_y", ctypes.c_void_p), ("d_z", ctypes.c_void_p), ("d_stream", ctypes.c_void_p),
                ("stream_bytes", ctypes.c_uint64), ("eb", ctypes.c_double), ("rel_eb", ctypes.c_double),
                ("rel_mode", ctypes.c_int32), ("seg_size", ctypes.c_uint32)]


class Completion(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("seg_size", ctypes.c_uint32), ("stream_bytes", ctypes.c_uint64),
                ("d_out", ctypes.c_void_p), ("eb", ctypes.c_double), ("queue_ms", ctypes.c_double),
                ("total_ms", ctypes.c_double), ("batch_size", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("batches", ctypes.c_uint64),
                ("arena_bytes", ctypes.c_uint64), ("arena_free_bytes", ctypes.c_uint64),
                ("queued", ctypes.c_uint32), ("in_flight", ctypes.c_uint32)]


class VerifyResult(ctypes.Structure):
    _fields_ = [("points", ctypes.c_uint64), ("over_bound", ctypes.c_uint64), ("over_bound_tol", ctypes.c_uint64),
                ("max_abs_err", ctypes.c_double * 3), ("mse", ctypes.c_double * 3),
                ("value_range", ctypes.c_double * 3), ("psnr", ctypes.c_double * 3),
                ("psnr_combined", ctypes.c_double)]


class DBatchItem(ctypes.Structure):
    """gpz_dbatch_item: one stream of a batched decompress."""
    _fields_ = [("d_stream", ctypes.c_void_p), ("stream_bytes", ctypes.c_uint64), ("float_bits", ctypes.c_uint32),
                ("dim", ctypes.c_uint32), ("n", ctypes.c_uint64), ("d_x", ctypes.c_void_p), ("d_y", ctypes.c_void_p),
                ("d_z", ctypes.c_void_p), ("out_capacity", ctypes.c_uint64)]

# name -> (restype, argtypes); the exported surface of include/gpz_b200.h
SIGNATURES = {
    "gpz_stream_bound": (_U64, [_U64, _U32, _U32]),
    "gpz_compress_scratch_bytes": (_U64, [_U64]),
    "gpz_decompress_scratch_bytes": (_U64, []),
    "gpz_compress_async": (ctypes.c_int, [ctypes.POINTER(Params), _VP, _VP, _VP, _VP, _U64, _VP, _U64, _VP]),
    "gpz_compress": (ctypes.c_int, [ctypes.POINTER(Params), _VP, _VP, _VP, _VP, _U64, _VP, _U64,
                                    ctypes.POINTER(Result), _VP]),
    "gpz_decompress_async": (ctypes.c_int, [_VP, _U64, _U32, _U32, _VP, _VP, _VP, _U64, _VP, _U64, _VP]),
    "gpz_decompress": (ctypes.c_int, [_VP, _U64, _U32, _U32, _VP, _VP, _VP, _U64, _VP, _U64,
                                      ctypes.POINTER(Result), _VP]),
    "gpz_result_get": (ctypes.c_int, [_VP, ctypes.POINTER(Result), _VP]),
    "gpz_result_post": (ctypes.c_int, [_VP, _VP, _VP]),
    "gpz_parse_header": (ctypes.c_int, [_VP, _U64, ctypes.POINTER(_U32), ctypes.POINTER(_U64),
                                        ctypes.POINTER(_U32), ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(_U32)]),
    "gpz_rel_to_abs": (ctypes.c_int, [_U32, _U32, _U64, _VP, _VP, _VP, ctypes.c_double, _VP, _U64,
                                      ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double), _VP]),
    "gpz_version": (ctypes.c_char_p, []),
    "gpz_compress_noalloc_max_points": (_U64, []),
    "gpz_compress_noalloc": (ctypes.c_int, [ctypes.POINTER(Params), _VP, _VP, _VP, _VP, _U64,
                                            ctypes.POINTER(Result), _VP]),
    "gpz_aos_to_soa": (ctypes.c_int, [_U32, _U32, _U64, _VP, _VP, _VP, _VP, _VP]),
    "gpz_soa_to_aos": (ctypes.c_int, [_U32, _U32, _U64, _VP, _VP, _VP, _VP, _VP]),
    "gpz_stream_size": (ctypes.c_int, [_VP, _U64, ctypes.POINTER(_U64), _VP]),
    "gpz_sample_minmax": (ctypes.c_int, [_U32, _U32, _U64, _U64, _U64, _VP, _VP, _VP, _VP, _U64,
                                         ctypes.POINTER(_U64), _VP]),
    "gpz_decide_seg": (ctypes.c_int, [_U32, _U32, ctypes.POINTER(_U64), _U32, ctypes.c_int32, ctypes.c_double,
                                      ctypes.c_double, _U32, ctypes.POINTER(_U32), ctypes.POINTER(_U32)]),
    "gpz_rel_abs_from_minmax": (ctypes.c_int, [_U32, ctypes.POINTER(ctypes.c_double), ctypes.c_double,
                                               ctypes.POINTER(ctypes.c_double)]),
    "gpz_strict_bound": (ctypes.c_int, [_U32, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                        ctypes.POINTER(ctypes.c_double)]),
    "gpz_batch_create": (ctypes.c_int, [ctypes.POINTER(BatchItem), _U32, ctypes.POINTER(_VP), ctypes.POINTER(_U32)]),
    "gpz_batch_launch": (ctypes.c_int, [_VP, _VP]),
    "gpz_batch_results": (ctypes.c_int, [_VP, ctypes.POINTER(Result), ctypes.POINTER(ctypes.c_double), _VP]),
    "gpz_batch_device_bytes": (_U64, [_VP]),
    "gpz_batch_destroy": (ctypes.c_int, [_VP]),
    "gpz_dbatch_create": (ctypes.c_int, [ctypes.POINTER(DBatchItem), _U32, ctypes.POINTER(_VP),
                                         ctypes.POINTER(_U32)]),
    "gpz_dbatch_launch": (ctypes.c_int, [_VP, _VP]),
    "gpz_dbatch_results": (ctypes.c_int, [_VP, ctypes.POINTER(Result), _VP]),
    "gpz_dbatch_destroy": (ctypes.c_int, [_VP]),
    "gpz_server_create": (ctypes.c_int, [ctypes.POINTER(ServerConfig), ctypes.POINTER(_VP)]),
    "gpz_server_submit": (ctypes.c_int, [_VP, ctypes.POINTER(Request), ctypes.POINTER(_U64)]),
    "gpz_server_wait": (ctypes.c_int, [_VP, _U64, ctypes.POINTER(Completion), _U32]),
    "gpz_server_release": (ctypes.c_int, [_VP, _U64]),
    "gpz_server_stats_get": (ctypes.c_int, [_VP, ctypes.POINTER(ServerStats)]),
    "gpz_server_destroy": (ctypes.c_int, [_VP]),
    "gpz_verify_scratch_bytes": (_U64, []),
    "gpz_selftest_lookback_timeout": (ctypes.c_int, [_U32, _VP, _U64, ctypes.POINTER(ctypes.c_int32), _VP]),
    "gpz_verify": (ctypes.c_int, [_U32, _U32, _U64, _VP, _VP, _VP, _VP, _VP, _VP, ctypes.c_double, _U32, _VP, _U64,
                                  ctypes.POINTER(VerifyResult), _VP]),
    "gpz_verify_bound": (ctypes.c_int, [_U32, _U32, _U64, _VP, _VP, _VP, _VP, _VP, _VP, ctypes.c_double, _U32,
                                        ctypes.c_double, _VP, _U64, ctypes.POINTER(VerifyResult), _VP]),
}

_lib = None


def build(force: bool = False) -> str:
    """Compiles the CUDA library in-tree for sm_100a (nvcc cross-compiles without a GPU)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", os.path.join(HERE, "csrc")], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C gpz_b200/csrc` "
                              "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(rc: int, what: str):
    if rc != GPZ_OK:
        raise GpzError(rc, what)


def _torch():
    import torch
    return torch


def _stream_ptr(stream):
    torch = _torch()
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


def _dtype_bits(t):
    torch = _torch()
    if t.dtype == torch.float32:
        return 32
    if t.dtype == torch.float64:
        return 64
    raise TypeError(f"coordinates must be float32 or float64, got {t.dtype}")


def stream_bound(n: int, dim: int, float_bits: int) -> int:
    return int(lib().gpz_stream_bound(n, dim, float_bits))


def compress_scratch_bytes(n: int) -> int:
    return int(lib().gpz_compress_scratch_bytes(n))


def make_params(n: int, dim: int, float_bits: int, eb: float, seg_size: int = 0, rel_mode: bool = False,
                rel_eb: float = 0.0, safe31: bool = False, strict: bool = False) -> Params:
    flags = (GPZ_FLAG_SAFE31 if safe31 else 0) | (GPZ_FLAG_STRICT_BOUND if strict else 0)
    return Params(float_bits=float_bits, dim=dim, n=n, eb=eb, rel_eb=rel_eb, rel_mode=1 if rel_mode else 0,
                  seg_size=seg_size, flags=flags, reserved=0)


def strict_bound(float_bits: int, eb: float, max_abs: float, max_range: float) -> float:
    """The bound GPZ_FLAG_STRICT_BOUND encodes with for a snapshot whose largest
    coordinate magnitude is max_abs and largest per-axis range max_range
    (gpz_strict_bound)."""
    out = ctypes.c_double()
    _check(lib().gpz_strict_bound(float_bits, eb, max_abs, max_range, ctypes.byref(out)), "gpz_strict_bound")
    return out.value


def compress_into(params: Params, x, y, z, out, scratch, stream=None, sync: bool = True):
    """Enqueues a compress of SoA tensors into the uint8 tensor `out` using the uint8 tensor
    `scratch`.  With sync=True returns the Result; otherwise returns None."""
    zp = z.data_ptr() if params.dim == 3 else None
    sp = _stream_ptr(stream)
    rc = lib().gpz_compress_async(ctypes.byref(params), x.data_ptr(), y.data_ptr(), zp, out.data_ptr(),
                                  out.numel(), scratch.data_ptr(), scratch.numel(), sp)
    _check(rc, "gpz_compress_async")
    if not sync:
        return None
    return result_get(scratch, stream)


def result_get(scratch, stream=None) -> Result:
    r = Result()
    rc = lib().gpz_result_get(scratch.data_ptr(), ctypes.byref(r), _stream_ptr(stream))
    _check(rc, "gpz_result_get")
    return r


def result_post(scratch, host_result, stream=None):
    """Enqueues a copy of the scratch's result into `host_result`, a pinned
    uint8 CPU tensor of at least ctypes.sizeof(Result) bytes, without a copy
    engine; read it with `Result.from_address(host_result.data_ptr())` after
    the stream has passed this point."""
    if host_result.device.type != "cpu" or not host_result.is_pinned() or host_result.numel() < ctypes.sizeof(Result):
        raise GpzError(GPZ_EINVAL, "gpz_result_post")
    _check(lib().gpz_result_post(scratch.data_ptr(), host_result.data_ptr(), _stream_ptr(stream)), "gpz_result_post")


def compress(x, y, z=None, eb: float = 0.0, seg_size: int = 0, rel_mode: bool = False, rel_eb: float = 0.0,
             safe31: bool = False, stream=None, strict: bool = False):
    """Compresses SoA CUDA tensors; returns (stream bytes as a uint8 CUDA tensor, Result)."""
    torch = _torch()
    dim = 3 if z is not None else 2
    bits = _dtype_bits(x)
    n = x.numel()
    p = make_params(n, dim, bits, eb, seg_size, rel_mode, rel_eb, safe31, strict)
    out = torch.empty(stream_bound(n, dim, bits), dtype=torch.uint8, device=x.device)
    scratch = torch.empty(compress_scratch_bytes(n), dtype=torch.uint8, device=x.device)
    r = compress_into(p, x, y, z if dim == 3 else x, out, scratch, stream)
    return out[: r.stream_bytes], r


def parse_header(host_bytes: bytes):
    buf = ctypes.create_string_buffer(bytes(host_bytes[:32]), 32)
    dim = _U32(); n = _U64(); bits = _U32(); eb = ctypes.c_double(); seg = _U32()
    rc = lib().gpz_parse_header(ctypes.cast(buf, _VP), min(len(host_bytes), 32), ctypes.byref(dim), ctypes.byref(n),
                                ctypes.byref(bits), ctypes.byref(eb), ctypes.byref(seg))
    _check(rc, "gpz_parse_header")
    return dict(dim=dim.value, n=n.value, float_bits=bits.value, eb=eb.value, seg=seg.value)


def decompress_into(d_stream, nbytes: int, float_bits: int, dim: int, x, y, z, scratch, stream=None,
                    sync: bool = True):
    zp = z.data_ptr() if dim == 3 else None
    rc = lib().gpz_decompress_async(d_stream.data_ptr(), nbytes, float_bits, dim, x.data_ptr(), y.data_ptr(), zp,
                                    x.numel(), scratch.data_ptr(), scratch.numel(), _stream_ptr(stream))
    _check(rc, "gpz_decompress_async")
    if not sync:
        return None
    r = result_get(scratch, stream)
    return r


def decompress(d_stream, header: dict | None = None, stream=None):
    """Decompresses a uint8 CUDA tensor holding a stream; returns (x, y, z) (z is None for 2D)."""
    torch = _torch()
    if header is None:
        header = parse_header(d_stream[:32].cpu().numpy().tobytes())
    dtype = torch.float32 if header["float_bits"] == 32 else torch.float64
    n, dim = header["n"], header["dim"]
    dev = d_stream.device
    x = torch.empty(n, dtype=dtype, device=dev)
    y = torch.empty(n, dtype=dtype, device=dev)
    z = torch.empty(n, dtype=dtype, device=dev) if dim == 3 else None
    scratch = torch.empty(int(lib().gpz_decompress_scratch_bytes()), dtype=torch.uint8, device=dev)
    decompress_into(d_stream, d_stream.numel(), header["float_bits"], dim, x, y, z if dim == 3 else x, scratch,
                    stream)
    return x, y, z


def rel_to_abs(x, y, z, rel: float, stream=None):
    """Relative -> absolute bound on the device, as the reference CLI computes it on the host.
    Returns (eb, [x_min, y_min, z_min, x_max, y_max, z_max])."""
    torch = _torch()
    dim = 3 if z is not None else 2
    bits = _dtype_bits(x)
    scratch = torch.empty(256, dtype=torch.uint8, device=x.device)
    eb = ctypes.c_double()
    mm = (ctypes.c_double * 6)()
    rc = lib().gpz_rel_to_abs(bits, dim, x.numel(), x.data_ptr(), y.data_ptr(), z.data_ptr() if z is not None else None,
                              rel, scratch.data_ptr(), 256, ctypes.byref(eb), mm, _stream_ptr(stream))
    _check(rc, "gpz_rel_to_abs")
    return eb.value, list(mm)


def verify(x, y, z, rx, ry, rz, eb: float, seg_size: int, stream=None, bound: float | None = None) -> "VerifyResult":
    """Per-point check of a reconstruction (stream order, as decompress
    returns it) against the original SoA tensors; eb and seg_size as in the
    stream header, `bound` the bound the errors are checked against (default
    eb; the stated bound for a strict-bound stream, whose header eb is below
    it)."""
    torch = _torch()
    dim = 3 if z is not None else 2
    scratch = torch.empty(int(lib().gpz_verify_scratch_bytes()), dtype=torch.uint8, device=x.device)
    res = VerifyResult()
    rc = lib().gpz_verify_bound(_dtype_bits(x), dim, x.numel(), x.data_ptr(), y.data_ptr(),
                                z.data_ptr() if dim == 3 else None, rx.data_ptr(), ry.data_ptr(),
                                rz.data_ptr() if dim == 3 else None, float(eb), int(seg_size),
                                float(eb if bound is None else bound), scratch.data_ptr(), scratch.numel(),
                                ctypes.byref(res), _stream_ptr(stream))
    _check(rc, "gpz_verify_bound")
    return res


# ---------------------------------------------------------------------------
# Mirror of the reference plugin interface.
# ---------------------------------------------------------------------------
@dataclass
class CudaConfig:
    """include/cudaCompress.cuh:16-40."""
    seg_size: int = 0
    adjusted_seg: bool = False
    dim: int = 3
    coordinate_num: int = 0
    error_mode: str = "abs"
    eb: float = 0.0
    rel_eb: float = 0.0
    float_bits: int = 32


class ICudaCompressor:
    """include/ICudaCompressor.cuh:6-17."""

    def compress(self, d_xyz, comp_data, comp_type: str = "none") -> int:  # returns comp_data_size
        raise NotImplementedError

    def decompress(self, x, y, z, d_compressed_data, nvcomp_type: str = "none") -> None:
        raise NotImplementedError

    def getConfig(self) -> CudaConfig:
        raise NotImplementedError


class _WarpCompressBase(ICudaCompressor):
    FLOAT_BITS = 32

    def __init__(self, cuda_config: CudaConfig | None = None):
        self.cuda_config = cuda_config if cuda_config is not None else CudaConfig(float_bits=self.FLOAT_BITS)

    def getConfig(self) -> CudaConfig:
        return self.cuda_config

    def compress(self, d_xyz, comp_data, comp_type: str = "none") -> int:
        """d_xyz: CUDA tensor holding x[N], y[N], z[N] back to back (z present even for 2D,
        src/main.cpp:283); comp_data: uint8 CUDA scratch of >= 4*N*sizeof(T) bytes
        (src/main.cpp:289-291).  The stream is written over d_xyz, as in
        src/cudaWarpCompress.cu:1669; returns the stream size."""
        torch = _torch()
        if comp_type not in ("", "none"):
            raise GpzError(GPZ_ENOTSUP, "nvcomp back-end")
        cfg = self.cuda_config
        n = cfg.coordinate_num
        v = d_xyz.view(torch.float32 if self.FLOAT_BITS == 32 else torch.float64)
        x, y, z = v[:n], v[n:2 * n], v[2 * n:3 * n]
        p = make_params(n, cfg.dim, self.FLOAT_BITS, cfg.eb, cfg.seg_size, cfg.error_mode == "rel", cfg.rel_eb)
        bound = stream_bound(n, cfg.dim, self.FLOAT_BITS)
        need = compress_scratch_bytes(n)
        cd = comp_data.view(torch.uint8)
        if cd.numel() >= bound + need + 256:
            out, scratch = cd[:bound], cd[cd.numel() - need - 255:]
            off = (256 - scratch.data_ptr() % 256) % 256
            scratch = scratch[off:off + need]
        else:
            out = torch.empty(bound, dtype=torch.uint8, device=d_xyz.device)
            scratch = torch.empty(need, dtype=torch.uint8, device=d_xyz.device)
        r = compress_into(p, x, y, z if cfg.dim == 3 else x, out, scratch)
        dst = d_xyz.view(torch.uint8)
        if r.stream_bytes > dst.numel():
            raise GpzError(GPZ_ENOSPACE, "compress (stream larger than the input buffer)")
        dst[: r.stream_bytes].copy_(out[: r.stream_bytes])
        cfg.seg_size = r.seg_size
        cfg.adjusted_seg = bool(r.adjusted) or cfg.adjusted_seg
        return int(r.stream_bytes)

    def decompress(self, x, y, z, d_compressed_data, nvcomp_type: str = "none") -> None:
        torch = _torch()
        if nvcomp_type not in ("", "none"):
            raise GpzError(GPZ_ENOTSUP, "nvcomp back-end")
        h = parse_header(d_compressed_data[:32].cpu().numpy().tobytes())
        scratch = torch.empty(256, dtype=torch.uint8, device=d_compressed_data.device)
        decompress_into(d_compressed_data, d_compressed_data.numel(), h["float_bits"], h["dim"], x, y,
                        z if h["dim"] == 3 else x, scratch)


class CudaWarpCompress(_WarpCompressBase):
    """include/cudaWarpCompress.cuh:11-39 (float32)."""
    FLOAT_BITS = 32


class CudaWarpCompressDouble(_WarpCompressBase):
    """include/cudaWarpCompressDouble.cuh:11-39 (float64)."""
    FLOAT_BITS = 64


class CompressorManager:
    """include/CompressorManager.h:9-28, src/CompressorManager.cpp:8-34."""

    def compressWarp(self, d_xyz, d_comp_data, nvcomp_type: str, compressor: ICudaCompressor) -> int:
        return compressor.compress(d_xyz, d_comp_data, nvcomp_type)

    def decompressWarp(self, x, y, z, d_compressed_data, decompressor: ICudaCompressor, nvcomp_type: str) -> None:
        decompressor.decompress(x, y, z, d_compressed_data, nvcomp_type)

    def decompressLoadParas(self, nvcomp_type: str, nvcomp_num: int, nvcomp_dim: int, float_bits_num: int,
                            h_compressed_data: bytes):
        """Returns (dim, num_points, float_bits)."""
        if nvcomp_type not in ("", "none"):
            return nvcomp_dim, nvcomp_num, float_bits_num
        h = parse_header(h_compressed_data)
        return h["dim"], h["n"], h["float_bits"]
