"""CPU-side checks of the CUDA library: it loads without a GPU, exports every
entry point that include/gpz_b200.h declares, and its host helpers behave."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import gpz_b200 as gz
from oracle import pyoracle as po

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "gpz_b200.h")).read()
    return sorted(set(re.findall(r"\b(gpz_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = gz.lib()
    declared = _declared()
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(gz.SIGNATURES), "Python signature table out of sync with the header"


def test_version_and_sizes():
    lib = gz.lib()
    assert b"sm_100a" in lib.gpz_version()
    n = 143_735_721
    G = (n + 1023) // 1024
    assert gz.compress_scratch_bytes(n) == 256 + 8 * G
    assert gz.stream_bound(n, 3, 32) == po.lib().gpzo_stream_bound(n, 3, 32)
    assert lib.gpz_decompress_scratch_bytes() == 256


def test_parse_header_matches_reference_layout():
    x, y, z = po.generate(0, 5000, 3, 0.0, 1.0, 3, np.float32)
    s = po.compress(x, y, z, 3, 1e-3, 4)
    h = gz.parse_header(s)
    assert h == dict(dim=3, n=5000, float_bits=32, eb=float(np.float32(1e-3)), seg=4)
    x, y, z = po.generate(0, 3000, 2, 0.0, 1.0, 3, np.float64)
    s = po.compress(x, y, None, 2, 1e-3, 2)
    assert gz.parse_header(s) == dict(dim=2, n=3000, float_bits=64, eb=1e-3, seg=2)
    with pytest.raises(gz.GpzError):
        gz.parse_header(b"\x05" + bytes(31))


def test_host_argument_errors_without_gpu():
    """Argument validation happens before any CUDA call."""
    lib = gz.lib()
    p = gz.make_params(100, 4, 32, 1e-3, 2)
    rc = lib.gpz_compress_async(ctypes.byref(p), 16, 16, 16, 16, 1 << 20, 256, 4096, None)
    assert rc == gz.GPZ_EINVAL
    p = gz.make_params(100, 3, 32, 1e-3, 0)  # abs mode without a segment size
    rc = lib.gpz_compress_async(ctypes.byref(p), 16, 16, 16, 16, 1 << 20, 256, 4096, None)
    assert rc == gz.GPZ_EINVAL
    rc = lib.gpz_decompress_async(16, 100, 16, 3, 16, 16, 16, 10, 256, 256, None)
    assert rc == gz.GPZ_EINVAL
    assert lib.gpz_result_post(None, 16, None) == gz.GPZ_EINVAL  # no scratch
    assert lib.gpz_result_post(16, None, None) == gz.GPZ_EINVAL  # no host result


@pytest.mark.parametrize("check", ["fastdiv_check", "transpose_check", "network_check", "bucket_check"])
def test_device_helpers_on_host(tmp_path, check):
    """Exact dividers, bit-plane transposes, register sorting networks and the
    bucket ranking's schedule of the kernels, compiled for the host and checked
    against plain arithmetic."""
    exe = tmp_path / check
    subprocess.run(["nvcc", "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", os.path.join(ROOT, "gpz_b200", "csrc"), "-I", os.path.join(ROOT, "include"),
                    "-o", str(exe), os.path.join(ROOT, "tests", "host", check + ".cu")], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "bad=0" in out.stdout
