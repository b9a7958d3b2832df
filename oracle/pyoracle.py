"""ctypes bindings to the CPU oracle (oracle/libgpz_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by ``bench.py``'s CPU-baseline / reference arm, always as the checker or
the timed CPU baseline, never on the product path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgpz_oracle.so")

_lib = None

u8p = ctypes.POINTER(ctypes.c_uint8)
u64p = ctypes.POINTER(ctypes.c_uint64)
u32p = ctypes.POINTER(ctypes.c_uint32)
f32p = ctypes.POINTER(ctypes.c_float)
f64p = ctypes.POINTER(ctypes.c_double)
intp = ctypes.POINTER(ctypes.c_int)


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.gpzo_stream_bound.restype = ctypes.c_uint64
        L.gpzo_stream_bound.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32]
        L.gpzo_rel_to_abs_f32.restype = ctypes.c_float
        L.gpzo_rel_to_abs_f32.argtypes = [f32p, f32p, f32p, ctypes.c_uint64, ctypes.c_float]
        L.gpzo_rel_to_abs_f64.restype = ctypes.c_double
        L.gpzo_rel_to_abs_f64.argtypes = [f64p, f64p, f64p, ctypes.c_uint64, ctypes.c_double]
        for t, tp, ft in (("f32", f32p, ctypes.c_float), ("f64", f64p, ctypes.c_double)):
            f = getattr(L, f"gpzo_seg_size_{t}")
            f.restype = ctypes.c_int
            f.argtypes = [tp, tp, tp, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
                          ctypes.c_int, ft, ft, ctypes.c_int, u32p, intp]
            f = getattr(L, f"gpzo_compress_{t}")
            f.restype = ctypes.c_int
            f.argtypes = [tp, tp, tp, ctypes.c_uint64, ctypes.c_uint32, ft, ctypes.c_uint32,
                          u8p, u64p, ctypes.c_int]
            f = getattr(L, f"gpzo_decompress_{t}")
            f.restype = ctypes.c_int
            f.argtypes = [u8p, ctypes.c_uint64, tp, tp, tp, ctypes.c_uint64, ctypes.c_int]
            f = getattr(L, f"gpzo_permutation_{t}")
            f.restype = ctypes.c_int
            f.argtypes = [tp, tp, tp, ctypes.c_uint64, ctypes.c_uint32, ft, ctypes.c_uint32, u64p]
            f = getattr(L, f"gpzo_generate_{t}")
            f.restype = None
            f.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_double,
                          ctypes.c_double, ctypes.c_uint64, tp, tp, tp]
        L.gpzo_parse_header.restype = ctypes.c_int
        L.gpzo_parse_header.argtypes = [u8p, ctypes.c_uint64, u32p, u64p, u32p,
                                        ctypes.POINTER(ctypes.c_double), u32p]
        L.gpzo_padding_mask.restype = ctypes.c_int
        L.gpzo_padding_mask.argtypes = [u8p, ctypes.c_uint64, u8p]
        L.gpzo_set_decode_fma.restype = None
        L.gpzo_set_decode_fma.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def _p(a, typ):
    if a is None:
        return None
    return a.ctypes.data_as(typ)


def _tp(dtype):
    return (f32p, "f32") if np.dtype(dtype) == np.float32 else (f64p, "f64")


class OracleError(RuntimeError):
    def __init__(self, code, what):
        super().__init__(f"oracle {what} failed with code {code}")
        self.code = code


def generate(kind: int, n: int, dim: int, lo: float, hi: float, seed: int, dtype=np.float32):
    """Deterministic synthetic SoA points: returns (x, y, z) (z is zeros for 2D)."""
    tp, t = _tp(dtype)
    x = np.empty(n, dtype); y = np.empty(n, dtype); z = np.zeros(n, dtype)
    getattr(lib(), f"gpzo_generate_{t}")(kind, n, dim, lo, hi, seed, _p(x, tp), _p(y, tp), _p(z, tp))
    return x, y, z


def rel_to_abs(x, y, z, rel: float) -> float:
    tp, t = _tp(x.dtype)
    return float(getattr(lib(), f"gpzo_rel_to_abs_{t}")(_p(x, tp), _p(y, tp), _p(z, tp), len(x), rel))


def seg_size(x, y, z, dim: int, seg_in: int, rel_mode: bool, rel_eb: float, eb: float,
             safe31: bool = False):
    """Returns (seg, adjusted) as computeSegSize leaves them in CudaConfig."""
    tp, t = _tp(x.dtype)
    seg = ctypes.c_uint32(0)
    adj = ctypes.c_int(0)
    rc = getattr(lib(), f"gpzo_seg_size_{t}")(
        _p(x, tp), _p(y, tp), _p(z, tp) if dim == 3 else None, len(x), dim, seg_in,
        int(rel_mode), rel_eb, eb, int(safe31), ctypes.byref(seg), ctypes.byref(adj))
    if rc:
        raise OracleError(rc, "seg_size")
    return seg.value, bool(adj.value)


def compress(x, y, z, dim: int, eb: float, seg: int, nthreads: int = 0) -> bytes:
    tp, t = _tp(x.dtype)
    n = len(x)
    bits = 32 if t == "f32" else 64
    out = np.empty(lib().gpzo_stream_bound(n, dim, bits), np.uint8)
    nb = ctypes.c_uint64(0)
    rc = getattr(lib(), f"gpzo_compress_{t}")(
        _p(x, tp), _p(y, tp), _p(z, tp) if dim == 3 else None, n, dim, eb, seg,
        _p(out, u8p), ctypes.byref(nb), nthreads)
    if rc:
        raise OracleError(rc, "compress")
    return out[: nb.value].tobytes()


def parse_header(stream: bytes):
    buf = np.frombuffer(stream, np.uint8)
    dim = ctypes.c_uint32(); n = ctypes.c_uint64(); bits = ctypes.c_uint32()
    eb = ctypes.c_double(); seg = ctypes.c_uint32()
    rc = lib().gpzo_parse_header(_p(buf, u8p), len(buf), ctypes.byref(dim), ctypes.byref(n),
                                 ctypes.byref(bits), ctypes.byref(eb), ctypes.byref(seg))
    if rc:
        raise OracleError(rc, "parse_header")
    return dict(dim=dim.value, n=n.value, float_bits=bits.value, eb=eb.value, seg=seg.value)


def decompress(stream: bytes, nthreads: int = 0):
    h = parse_header(stream)
    dtype = np.float32 if h["float_bits"] == 32 else np.float64
    tp, t = _tp(dtype)
    n = h["n"]
    x = np.zeros(n, dtype); y = np.zeros(n, dtype); z = np.zeros(n, dtype)
    buf = np.frombuffer(stream, np.uint8)
    rc = getattr(lib(), f"gpzo_decompress_{t}")(_p(buf, u8p), len(buf), _p(x, tp), _p(y, tp),
                                                 _p(z, tp), n, nthreads)
    if rc:
        raise OracleError(rc, "decompress")
    return x, y, z


def permutation(x, y, z, dim: int, eb: float, seg: int):
    tp, t = _tp(x.dtype)
    perm = np.empty(len(x), np.uint64)
    rc = getattr(lib(), f"gpzo_permutation_{t}")(
        _p(x, tp), _p(y, tp), _p(z, tp) if dim == 3 else None, len(x), dim, eb, seg, _p(perm, u64p))
    if rc:
        raise OracleError(rc, "permutation")
    return perm


def padding_mask(stream: bytes):
    buf = np.frombuffer(stream, np.uint8)
    mask = np.zeros(len(buf), np.uint8)
    rc = lib().gpzo_padding_mask(_p(buf, u8p), len(buf), _p(mask, u8p))
    if rc:
        raise OracleError(rc, "padding_mask")
    return mask


def set_decode_fma(on: bool) -> None:
    lib().gpzo_set_decode_fma(int(on))
