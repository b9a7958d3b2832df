"""Failure detection of the placement look-back, tested without a fault: a
wait on a predecessor that never publishes runs out after its poll limit,
the kernel records GPZ_ETIMEOUT and returns, and the context stays usable
(a compress right afterwards is correct)."""
import ctypes
import time

import numpy as np
import pytest

import gpz_b200 as gz


def test_selftest_rejects_bad_arguments_before_touching_the_gpu():
    st = ctypes.c_int32(-1)
    assert gz.lib().gpz_selftest_lookback_timeout(0, 0x1000, 4096, ctypes.byref(st), None) == gz.GPZ_EINVAL
    assert gz.lib().gpz_selftest_lookback_timeout(1 << 23, 0x1000, 4096, ctypes.byref(st), None) == gz.GPZ_EINVAL
    assert gz.lib().gpz_selftest_lookback_timeout(10, 0x1000, 16, ctypes.byref(st), None) == gz.GPZ_ENOSPACE


@pytest.mark.gpu
def test_lookback_wait_runs_out_and_the_context_survives():
    import torch
    from oracle import pyoracle as po
    scratch = torch.empty(gz.compress_scratch_bytes(2048), dtype=torch.uint8, device="cuda")
    st = ctypes.c_int32(-1)
    t0 = time.perf_counter()
    rc = gz.lib().gpz_selftest_lookback_timeout(1 << 12, scratch.data_ptr(), scratch.numel(), ctypes.byref(st),
                                                gz._stream_ptr(None))
    assert rc == gz.GPZ_OK and st.value == gz.GPZ_ETIMEOUT
    assert time.perf_counter() - t0 < 30.0
    x, y, z = po.generate(1, 20_000, 3, 0.0, 100.0, 5, np.float32)
    eb = po.rel_to_abs(x, y, z, 1e-4)
    seg, _ = po.seg_size(x, y, z, 3, 0, True, float(np.float32(1e-4)), eb)
    tx, ty, tz = (torch.from_numpy(a).cuda() for a in (x, y, z))
    s, r = gz.compress(tx, ty, tz, eb=eb, rel_mode=True, rel_eb=float(np.float32(1e-4)))
    assert r.status == 0 and s.cpu().numpy().tobytes() == po.compress(x, y, z, 3, eb, seg)
