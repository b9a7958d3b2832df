"""Per-point verification (gpz_verify): the device pairing of reconstructed
and original points matches the oracle's permutation, the error statistics
match a host computation over that pairing, and a planted error is found."""
import numpy as np
import pytest

import gpz_b200 as gz


@pytest.mark.gpu
@pytest.mark.parametrize("kind,n,dim,bits,rel", [(1, 100_003, 3, 32, 1e-4), (0, 65_536, 2, 64, 1e-5),
                                                 (2, 30_000, 3, 64, 1e-5), (1, 1025, 3, 32, 1e-3)])
def test_verify_matches_a_host_check_over_the_oracle_pairing(kind, n, dim, bits, rel):
    import torch
    from oracle import pyoracle as po
    dt = np.float32 if bits == 32 else np.float64
    x, y, z = po.generate(kind, n, dim, 0.0, 500.0, 21, dt)
    tx, ty, tz = (torch.from_numpy(a.copy()).cuda() for a in (x, y, z))
    tz = tz if dim == 3 else None
    eb, _ = gz.rel_to_abs(tx, ty, tz, rel)
    s, r = gz.compress(tx, ty, tz, eb=eb, rel_mode=True, rel_eb=rel)
    rx, ry, rz = gz.decompress(s)
    h = gz.parse_header(s[:32].cpu().numpy().tobytes())
    v = gz.verify(tx, ty, tz, rx, ry, rz, h["eb"], h["seg"])
    # host: pair position s with original perm[s] (the oracle's encoder order)
    perm = po.permutation(x, y, z, dim, dt(h["eb"]), h["seg"])
    orig = [x, y, z][:dim]
    rec = [t.cpu().numpy() for t in (rx, ry, rz)[:dim]]
    assert v.points == n
    over = np.zeros(n, bool)
    over_tol = np.zeros(n, bool)
    for d in range(dim):
        e = np.abs(orig[d][perm].astype(np.float64) - rec[d].astype(np.float64))
        e_t = np.abs(orig[d][perm] - rec[d])  # in the point type, as the kernel computes it
        over |= ~(e_t <= dt(h["eb"]))
        over_tol |= ~(e_t <= dt(1.01 if bits == 64 else np.float32(1.01)) * dt(h["eb"]))
        assert v.max_abs_err[d] == float(e_t.max())
        assert v.mse[d] == pytest.approx(float(np.mean(e_t.astype(np.float64) ** 2)), rel=1e-9, abs=1e-300)
        assert v.value_range[d] == float(orig[d].max()) - float(orig[d].min())
    assert v.over_bound == int(over.sum())
    assert v.over_bound_tol == int(over_tol.sum())
    # the bound holds unless the reference's 31-bit block-id mask fired
    # (id_overflow: the lattice float64 case at rel 1e-5)
    assert v.over_bound_tol == 0 or r.id_overflow


@pytest.mark.gpu
def test_verify_finds_a_planted_error():
    import torch
    from oracle import pyoracle as po
    x, y, z = (torch.from_numpy(a.copy()).cuda() for a in po.generate(1, 50_000, 3, 0.0, 100.0, 4, np.float32))
    eb, _ = gz.rel_to_abs(x, y, z, 1e-4)
    s, _ = gz.compress(x, y, z, eb=eb, rel_mode=True, rel_eb=1e-4)
    rx, ry, rz = gz.decompress(s)
    h = gz.parse_header(s[:32].cpu().numpy().tobytes())
    base = gz.verify(x, y, z, rx, ry, rz, h["eb"], h["seg"])
    ry[12_345] += 10 * h["eb"]
    bad = gz.verify(x, y, z, rx, ry, rz, h["eb"], h["seg"])
    assert bad.over_bound_tol == base.over_bound_tol + 1
    assert bad.max_abs_err[1] > 9 * h["eb"]
