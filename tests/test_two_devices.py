"""Two GPUs in one process: the launch configuration (SM count, raised
shared-memory attribute, resident CTAs per SM) is kept per device, so a
compress on one device must not leave another device unconfigured.  The same
snapshot is compressed and decompressed on device 0, device 1, then device 0
again; every stream equals the oracle's and every reconstruction is
bit-identical.  Skipped where fewer than two GPUs are visible."""
import numpy as np
import pytest

from oracle import pyoracle as po

torch = pytest.importorskip("torch")

import gpz_b200 as gz  # noqa: E402


@pytest.mark.gpu
def test_compress_and_decompress_on_two_devices():
    if not torch.cuda.is_available() or torch.cuda.device_count() < 2:
        pytest.skip("needs two visible GPUs")
    x, y, z = po.generate(1, 300_000, 3, 0.0, 1000.0, 52, np.float32)
    eb = float(np.float32(po.rel_to_abs(x, y, z, 1e-4)))
    seg, _ = po.seg_size(x, y, z, 3, 0, True, float(np.float32(1e-4)), eb)
    ref = po.compress(x, y, z, 3, eb, seg)
    recon = []
    for dev in (0, 1, 0):
        with torch.cuda.device(dev):
            t = [torch.from_numpy(a).to(f"cuda:{dev}") for a in (x, y, z)]
            s, r = gz.compress(*t, eb=eb, rel_mode=True, rel_eb=float(np.float32(1e-4)))
            assert r.status == 0
            assert s.cpu().numpy().tobytes() == ref
            dx, dy, dz = gz.decompress(s)
            recon.append(np.concatenate([a.cpu().numpy() for a in (dx, dy, dz)]).view(np.uint8))
    assert all(np.array_equal(recon[0], o) for o in recon[1:])
