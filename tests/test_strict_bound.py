"""Strict-bound mode (GPZ_FLAG_STRICT_BOUND, an extension): every finite point
reconstructs within the stated bound.

The reference reconstructs min + (2q+1)*eb in the float type
(src/cudaWarpCompress.cu:971-1007), so points can land a few ulps past eb;
its verifier tolerates 1.01*eb (src/utils.cu:28).  In strict mode the codec
encodes with eb' = eb - u*(3*R + 2*M + 4*eb) (M = largest coordinate
magnitude, R = largest per-axis range, u = 2^-24 / 2^-53), computed on the
device; the stream is an ordinary GPZ
stream whose header carries eb', so the CPU oracle given eb' must produce the
same bytes.
"""
import numpy as np
import pytest

from oracle import pyoracle as po

torch = pytest.importorskip("torch")

import gpz_b200 as gz  # noqa: E402


def test_strict_bound_host_formula():
    """gpz_strict_bound: eb' = eb - u*(3R + 2M + 4eb), rounded down to the float type."""
    e = gz.strict_bound(32, 0.1, 1000.0, 999.0)
    assert e < np.float32(0.1) and e == float(np.float32(e))
    m = 2.0 ** -24 * (3 * 999.0 + 2 * 1000.0 + 0.4)
    assert m <= 0.1 - e < m + 1e-8
    e64 = gz.strict_bound(64, 1e-5, 369.0, 368.0)
    assert 1e-5 - e64 >= 2.0 ** -53 * (3 * 368.0 + 2 * 369.0) and e64 > 0
    with pytest.raises(gz.GpzError):
        gz.strict_bound(32, 1e-6, 1e6, 1e6)  # no positive bound is left


CASES = [
    # kind, n, dim, bits, lo, hi, seed, mode, e, seg
    (1, 300_000, 3, 32, 0.0, 1000.0, 41, "rel", 1e-4, 0),
    (1, 300_000, 3, 32, 0.0, 1000.0, 42, "abs", 1e-3, 32),
    (0, 200_000, 3, 32, -300.0, 700.0, 43, "abs", 7e-3, 8),
    (2, 150_000, 3, 64, 0.0, 0.05, 44, "rel", 1e-5, 0),
    (2, 100_000, 2, 64, 0.0, 0.05, 45, "rel", 1e-5, 0),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=[f"{c[0]}-{c[1]}-{c[2]}d-f{c[3]}-{c[7]}{c[8]}" for c in CASES])
def test_strict_mode_holds_the_bound_and_matches_the_oracle(case):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    kind, n, dim, bits, lo, hi, seed, mode, e, seg_in = case
    dt = np.float32 if bits == 32 else np.float64
    x, y, z = po.generate(kind, n, dim, lo, hi, seed, dt)
    typed = (lambda v: float(np.float32(v))) if bits == 32 else float
    eb = typed(po.rel_to_abs(x, y, z if dim == 3 else None, e) if mode == "rel" else e)
    tx, ty = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    tz = torch.from_numpy(z).cuda() if dim == 3 else None
    kw = dict(eb=eb, seg_size=seg_in, rel_mode=mode == "rel", rel_eb=typed(e))
    s, r = gz.compress(tx, ty, tz, strict=True, **kw)
    assert r.status == 0
    host = s.cpu().numpy().tobytes()
    hdr = gz.parse_header(host[:32])
    axes = (x, y, z) if dim == 3 else (x, y)
    M = max(float(np.nanmax(np.abs(a))) for a in axes)
    R = max(float(np.nanmax(a)) - float(np.nanmin(a)) for a in axes)
    eb_s = gz.strict_bound(bits, eb, M, R)
    assert hdr["eb"] == eb_s < eb
    # the same stream from the oracle given eb' (SAFE31 rules for the segment size)
    seg, adj = po.seg_size(x, y, z, dim, seg_in, mode == "rel", typed(e), eb_s, True)
    assert (r.seg_size, bool(r.adjusted)) == (seg, adj)
    assert host == po.compress(x, y, z, dim, eb_s, seg)
    # every point within the stated bound
    dx, dy, dz = gz.decompress(s)
    v = gz.verify(tx, ty, tz, dx, dy, dz, eb_s, r.seg_size, bound=eb)
    assert v.over_bound == 0 and v.over_bound_tol == 0, (v.over_bound, list(v.max_abs_err))
    assert max(v.max_abs_err[:dim]) <= eb


@pytest.mark.gpu
def test_default_mode_overshoots_where_strict_mode_does_not():
    """On clustered float32 data at rel 1e-4 the reference-identical default
    mode puts points just past eb (float rounding of the reconstruction);
    strict mode does not."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    x, y, z = po.generate(1, 1_000_000, 3, 0.0, 1000.0, 46, np.float32)
    eb = float(np.float32(po.rel_to_abs(x, y, z, 1e-4)))
    tx, ty, tz = (torch.from_numpy(a).cuda() for a in (x, y, z))
    over = {}
    for strict in (False, True):
        s, r = gz.compress(tx, ty, tz, eb=eb, rel_mode=True, rel_eb=float(np.float32(1e-4)), strict=strict)
        dx, dy, dz = gz.decompress(s)
        hdr = gz.parse_header(s[:32].cpu().numpy().tobytes())
        over[strict] = gz.verify(tx, ty, tz, dx, dy, dz, hdr["eb"], r.seg_size, bound=eb).over_bound
    assert over[False] > 0 and over[True] == 0, over
