"""Full-size parity: every headline workload, compressed on the GPU, against
the reference's own stream bytes (SHA-256 recorded from the reference codec
built from its sources, tests/golden/make_golden.py --full).

Workloads (tests/golden/full_size.json):
* 143,735,721 clustered float32 3D points at rel 1e-4 (automatic segment
  size) and at abs 1e-3 with segment size 32 (the reference doubles it to
  512, src/cudaWarpCompress.cu:1532-1554);
* 200,000,000 float64 3D points of a jittered FCC lattice at rel 1e-5;
* 100,000,000 float64 2D points of a jittered square lattice at rel 1e-5.

Streams must be byte-identical (at these sizes the reference's scratch is
zero-filled, so even its padding bytes are defined).  Reconstructions are
compared with the reference decoder's output where that decoder can run
(it writes out of bounds on chunks with 1024 unique blocks, see
oracle/ref_harness.cu) and otherwise with the CPU oracle, bit for bit.
"""
import hashlib
import json
import os
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import gpz_b200 as gz  # noqa: E402
from oracle import pyoracle as po  # noqa: E402

GOLD = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, GOLD)
import make_golden as mg  # noqa: E402

FULL = json.load(open(os.path.join(GOLD, "full_size.json")))["fixtures"]


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    gz.lib()


def _typed(bits, v):
    return float(np.float32(v)) if bits == 32 else float(v)


@pytest.mark.parametrize("f", FULL, ids=[f["name"] for f in FULL])
def test_full_size_stream_is_the_references(f):
    assert "stream_sha256" in f, f.get("compress_error")
    n, dim, bits = f["n"], f["dim"], f["bits"]
    x, y, z = mg.full_input(f["workload"], n)
    eb = mg.full_eb(x, y, z, dim, bits, f["mode"], f["e"])
    assert eb == f["eb"]
    dev = [torch.from_numpy(a).cuda() for a in ((x, y, z) if dim == 3 else (x, y))]
    del x, y, z
    s, r = gz.compress(dev[0], dev[1], dev[2] if dim == 3 else None, eb=_typed(bits, eb), seg_size=f["seg_in"],
                       rel_mode=f["mode"] == "rel", rel_eb=_typed(bits, f["e"]))
    assert r.status == 0
    assert (r.seg_size, bool(r.adjusted)) == (f["seg"], f["adjusted"])
    assert r.stream_bytes == f["bytes"]
    host = s.cpu().numpy()
    assert mg.sha_array(host) == f["stream_sha256"], "stream differs from the reference's"
    del dev
    rec = gz.decompress(s)
    del s
    axes = [t.cpu().numpy() for t in rec[:dim]]
    del rec
    torch.cuda.empty_cache()
    if "decoded_sha256" in f:
        assert mg.sha_array(*axes) == f["decoded_sha256"], "reconstruction differs from the reference decoder's"
    else:
        ox, oy, oz = po.decompress(host.tobytes())
        for a, b in zip(axes, (ox, oy, oz)):
            assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), "reconstruction differs from the oracle's"
