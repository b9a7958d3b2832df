"""gpz_compress_noalloc, the allocation-free compress entry point, through the C ABI.

Some callers cannot allocate device memory themselves: a codec plugin inside an
application that owns the whole device-memory budget and only lends it input
and output buffers, or a latency-critical path that cannot take cudaMalloc's
implicit device synchronisation.  gpz_compress_noalloc serves them by taking
its scratch from a fixed array inside the library.  Every call reuses that one
array, so these tests check that its streams equal the regular entry point's
(gpz_compress with caller-provided scratch) on consecutive calls, and that
inputs beyond the array's capacity are refused up front.

Kept in a file that pytest collects last; it also passes on its own.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import gpz_b200 as gz  # noqa: E402
from oracle import pyoracle as po  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    gz.lib()


def _case(kind, n, dim, bits, lo, hi, seed):
    dt = np.float32 if bits == 32 else np.float64
    x, y, z = po.generate(kind, n, dim, lo, hi, seed, dt)
    t = [torch.from_numpy(a.copy()).cuda() for a in (x, y, z)]
    return t


def _regular(p, x, y, z):
    """Stream from the regular entry point, scratch allocated by the caller."""
    out = torch.empty(gz.stream_bound(p.n, p.dim, p.float_bits), dtype=torch.uint8, device="cuda")
    scratch = torch.empty(gz.compress_scratch_bytes(p.n), dtype=torch.uint8, device="cuda")
    r = gz.Result()
    rc = gz.lib().gpz_compress(ctypes.byref(p), x.data_ptr(), y.data_ptr(), z.data_ptr() if p.dim == 3 else None,
                               out.data_ptr(), out.numel(), scratch.data_ptr(), scratch.numel(), ctypes.byref(r),
                               None)
    assert rc == gz.GPZ_OK
    return out[: r.stream_bytes].cpu().numpy().tobytes(), r


def _noalloc(p, x, y, z):
    out = torch.empty(gz.stream_bound(p.n, p.dim, p.float_bits), dtype=torch.uint8, device="cuda")
    r = gz.Result()
    rc = gz.lib().gpz_compress_noalloc(ctypes.byref(p), x.data_ptr(), y.data_ptr(),
                                       z.data_ptr() if p.dim == 3 else None, out.data_ptr(), out.numel(),
                                       ctypes.byref(r), None)
    assert rc == gz.GPZ_OK, gz.ERRORS.get(rc, rc)
    return out[: r.stream_bytes].cpu().numpy().tobytes(), r


def test_noalloc_matches_regular_entry_point_on_consecutive_calls():
    a = _case(1, 1_000_003, 3, 32, 0.0, 1000.0, 101)
    b = _case(0, 300_001, 2, 64, -10.0, 10.0, 102)
    pa = gz.make_params(a[0].numel(), 3, 32, float(np.float32(0.1)), 0, True, float(np.float32(1e-4)))
    pb = gz.make_params(b[0].numel(), 2, 64, 1e-3, 8, False, 0.0)
    ref_a, ra = _regular(pa, *a)
    ref_b, rb = _regular(pb, *b)
    # two calls in a row on the shared array, different sizes and types, then the first again
    got_a, ga = _noalloc(pa, *a)
    got_b, gb = _noalloc(pb, *b)
    got_a2, ga2 = _noalloc(pa, *a)
    assert got_a == ref_a and (ga.seg_size, ga.status) == (ra.seg_size, 0)
    assert got_b == ref_b and (gb.seg_size, gb.status) == (rb.seg_size, 0)
    assert got_a2 == ref_a


def test_noalloc_refuses_inputs_beyond_its_fixed_scratch():
    lim = int(gz.lib().gpz_compress_noalloc_max_points())
    assert lim == ((4 << 20) - 256) // 8 * 1024
    dummy = torch.zeros(16, dtype=torch.float32, device="cuda")
    out = torch.empty(1024, dtype=torch.uint8, device="cuda")
    p = gz.make_params(lim + 1, 3, 32, 0.1, 32)
    r = gz.Result()
    rc = gz.lib().gpz_compress_noalloc(ctypes.byref(p), dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(),
                                       out.data_ptr(), out.numel(), ctypes.byref(r), None)
    assert rc == gz.GPZ_ELIMIT
    torch.cuda.synchronize()
