"""GPU parity: the sm_100a codec (through the C ABI) against the CPU oracle and
the reference's own golden streams.

Integer / byte work is bit-exact: streams must equal the oracle's byte for
byte (padding included: both write zeros) and reconstructions must be
identical floats.  The oracle itself is pinned to the reference in
tests/test_oracle_golden.py.
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

FIX = json.load(open(os.path.join(GOLD, "cases.json")))["fixtures"]


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    gz.lib()


def _t(a):
    a = np.ascontiguousarray(a)
    return torch.from_numpy(a if a.flags.writeable else a.copy()).cuda()


def _typed(bits, v):
    return float(np.float32(v)) if bits == 32 else float(v)


def _oracle_case(x, y, z, dim, bits, mode, e, seg_in, safe31=False):
    eb = po.rel_to_abs(x, y, z if dim == 3 else None, e) if mode == "rel" else e
    ebT, relT = _typed(bits, eb), _typed(bits, e)
    seg, adj = po.seg_size(x, y, z, dim, seg_in, mode == "rel", relT, ebT, safe31)
    return ebT, relT, seg, adj, po.compress(x, y, z, dim, ebT, seg)


def _gpu_compress(x, y, z, dim, ebT, seg_in, mode, relT, safe31=False):
    s, r = gz.compress(_t(x), _t(y), _t(z) if dim == 3 else None, eb=ebT, seg_size=seg_in,
                       rel_mode=(mode == "rel"), rel_eb=relT, safe31=safe31)
    return s.cpu().numpy().tobytes(), r


def _check_roundtrip(stream, dim, bits):
    dx, dy, dz = gz.decompress(_t(np.frombuffer(stream, np.uint8)))
    ox, oy, oz = po.decompress(stream)
    assert np.array_equal(dx.cpu().numpy().view(np.uint8), ox.view(np.uint8))
    assert np.array_equal(dy.cpu().numpy().view(np.uint8), oy.view(np.uint8))
    if dim == 3:
        assert np.array_equal(dz.cpu().numpy().view(np.uint8), oz.view(np.uint8))
    return dx, dy, dz


def run_case(kind, n, dim, bits, lo, hi, seed, mode, e, seg_in, special=None, safe31=False):
    x, y, z = mg.make_input(kind, n, dim, bits, lo, hi, seed, special)
    return run_arrays(x, y, z, dim, bits, mode, e, seg_in, safe31)


def run_arrays(x, y, z, dim, bits, mode, e, seg_in, safe31=False):
    ebT, relT, seg, adj, s_o = _oracle_case(x, y, z, dim, bits, mode, e, seg_in, safe31)
    s_g, r = _gpu_compress(x, y, z, dim, ebT, seg_in, mode, relT, safe31)
    assert r.status == 0
    assert (r.seg_size, bool(r.adjusted)) == (seg, adj)
    assert r.stream_bytes == len(s_o)
    if s_g != s_o:
        a, b = np.frombuffer(s_g, np.uint8), np.frombuffer(s_o, np.uint8)
        bad = np.nonzero(a != b)[0]
        pytest.fail(f"stream differs from the oracle at {len(bad)} bytes, first {bad[:8].tolist()}")
    _check_roundtrip(s_g, dim, bits)
    return s_g


@pytest.mark.parametrize("f", FIX, ids=[f["name"] for f in FIX])
def test_golden_case_bit_exact(f):
    s = run_case(f["kind"], f["n"], f["dim"], f["bits"], f["lo"], f["hi"], f["seed"], f["mode"], f["e"],
                 f["seg_in"], f["special"])
    # and against the reference's own bytes
    assert len(s) == f["bytes"]
    if hashlib.sha256(s).hexdigest() == f["stream_sha256"]:
        return
    if "stream_file" in f:
        # the reference leaves section padding unwritten (stale scratch): mask it
        ref = np.frombuffer(open(os.path.join(GOLD, f["stream_file"]), "rb").read(), np.uint8)
        ours = np.frombuffer(s, np.uint8)
        mask = po.padding_mask(ref)
        diff = np.nonzero(ours != ref)[0]
        assert np.all(mask[diff] == 1), f"non-padding bytes differ at {diff[mask[diff] == 0][:8]}"
        assert np.all(ours[mask == 1] == 0)
    else:
        # stored as a hash only: below ~0.7M points the reference's padding
        # holds its sampling temporaries, so the hashes may differ there; its
        # own reconstruction then pins every other byte
        assert "decoded_sha256" in f, "stream differs from the reference's and no reconstruction pins it"
        dx, dy, dz = gz.decompress(_t(np.frombuffer(s, np.uint8)))
        axes = (dx, dy, dz if dz is not None else torch.zeros_like(dx))
        dec = b"".join(t.cpu().numpy().tobytes() for t in axes)
        assert hashlib.sha256(dec).hexdigest() == f["decoded_sha256"]


@pytest.mark.parametrize("f", [f for f in FIX if "stream_file" in f], ids=[f["name"] for f in FIX if "stream_file" in f])
def test_decodes_reference_stream(f):
    """Cross-decode: the GPU decoder reads the reference's own stream bytes."""
    ref = open(os.path.join(GOLD, f["stream_file"]), "rb").read()
    dx, dy, dz = _check_roundtrip(ref, f["dim"], f["bits"])
    if "decoded_file" in f:
        dec = open(os.path.join(GOLD, f["decoded_file"]), "rb").read()
        ours = b"".join(t.cpu().numpy().tobytes() for t in (dx, dy, dz if dz is not None else torch.zeros_like(dx)))
        assert ours == dec


EDGE = [
    # kind, n, dim, bits, lo, hi, seed, mode, e, seg
    (0, 1, 3, 32, 0.0, 100.0, 1, "abs", 1e-2, 4),
    (0, 2, 2, 32, 0.0, 100.0, 2, "abs", 1e-2, 4),
    (0, 31, 3, 64, 0.0, 100.0, 3, "abs", 1e-2, 8),
    (0, 1023, 3, 32, 0.0, 100.0, 4, "rel", 1e-4, 0),
    (0, 1024, 3, 32, 0.0, 100.0, 5, "rel", 1e-4, 0),
    (0, 1025, 2, 32, 0.0, 100.0, 6, "rel", 1e-3, 0),
    (0, 2047, 3, 64, -5.0, 5.0, 7, "rel", 1e-4, 0),
    (0, 65543, 3, 32, 0.0, 100.0, 8, "rel", 1e-4, 0),
    (0, 65543, 2, 64, 0.0, 100.0, 9, "rel", 1e-5, 0),
    (0, 40000, 3, 32, 0.0, 1.0, 10, "abs", 1e-3, 1),
    (0, 40000, 3, 32, 0.0, 1.0, 11, "abs", 1e-3, 2),
    (0, 40000, 3, 32, 0.0, 1.0, 12, "abs", 1e-3, 1024),
    (0, 40000, 3, 32, 0.0, 1.0, 13, "abs", 1e-3, 6),    # not a power of two: reference arithmetic kept
    (0, 40000, 3, 64, 0.0, 1.0, 14, "abs", 1e-4, 64),
    (1, 300000, 3, 32, 0.0, 1000.0, 15, "rel", 1e-4, 0),
    (1, 300000, 3, 32, 0.0, 1000.0, 16, "abs", 1e-3, 32),
    (2, 100000, 3, 64, 0.0, 0.05, 17, "rel", 1e-5, 0),
    (2, 50000, 2, 64, 0.0, 0.05, 18, "rel", 1e-5, 0),
    (0, 20000, 3, 32, 0.0, 1e-3, 19, "abs", 1.0, 2),     # everything in one block
    # wide composites (id range above 2^22): the bucket ranking, on clustered
    # data (crowded buckets) and uniform data
    (1, 200000, 3, 32, 0.0, 1000.0, 20, "rel", 1e-5, 0),
    (1, 120000, 3, 64, 0.0, 1000.0, 21, "rel", 1e-5, 0),
    (0, 100000, 3, 64, 0.0, 1000.0, 22, "abs", 1e-4, 1),   # rel positions 0 bits, ids 31 bits
]


@pytest.mark.parametrize("case", EDGE, ids=[f"{c[0]}-{c[1]}-{c[2]}d-f{c[3]}-{c[7]}{c[8]}-s{c[9]}" for c in EDGE])
def test_edge_cases_bit_exact(case):
    run_case(*case)


@pytest.mark.parametrize("mode,e,seg", [("abs", 0.05, 8), ("rel", 1e-4, 0)])
@pytest.mark.parametrize("bits,dim", [(32, 3), (32, 2), (64, 3), (64, 2)])
def test_nan_points_bit_exact(bits, dim, mode, e, seg):
    """NaN coordinates are ignored by the chunk min/max and quantize to 0 (the
    GPU's min/max and saturating conversion); signed zeros order -0.0 below
    +0.0.  Covered: NaNs scattered over whole chunks, a chunk whose first
    point is NaN, a short last chunk whose first point (the one its unused
    slots repeat) is NaN, and a chunk whose x axis is NaN throughout."""
    dtype = np.float32 if bits == 32 else np.float64
    n = 6 * 1024 + 300
    x, y, z = po.generate(0, n, dim, 0.0, 100.0, 21, dtype)
    rng = np.random.default_rng(5)
    for a in (x, y, z):
        a[rng.choice(n, 60, replace=False)] = np.nan
    x[1024] = np.nan                  # first point of chunk 1
    y[6 * 1024] = np.nan              # first point of the short last chunk
    x[6 * 1024 + 1] = -0.0
    x[6 * 1024 + 2] = 0.0
    x[3 * 1024:4 * 1024] = np.nan     # chunk 3: no x value at all
    if dim == 2:
        z[:] = 0
    run_arrays(x, y, z, dim, bits, mode, e, seg)


@pytest.mark.parametrize("heavy", [17, 90, 300, 1023])
def test_heavy_duplicate_block(heavy):
    """A dominant cluster: `heavy` points of every chunk share one block while the
    rest spread over the box, so one ranking bucket is large and is sorted by a warp."""
    n = 8 * 1024 + 77
    x, y, z = po.generate(0, n, 3, 0.0, 1000.0, 31 + heavy, np.float32)
    rng = np.random.default_rng(heavy)
    for c in range(0, n, 1024):
        m = min(heavy, n - c)
        sel = c + rng.choice(min(1024, n - c), m, replace=False)
        x[sel] = 500.0 + rng.random(m).astype(np.float32) * 0.05
        y[sel] = 250.0 + rng.random(m).astype(np.float32) * 0.05
        z[sel] = 750.0 + rng.random(m).astype(np.float32) * 0.05
    for seg in (4, 32):
        s_o = po.compress(x, y, z, 3, float(np.float32(0.1)), seg)
        s_g, r = _gpu_compress(x, y, z, 3, float(np.float32(0.1)), seg, "abs", 0.0)
        assert s_g == s_o
        _check_roundtrip(s_g, 3, 32)


def test_fallback_sort_outlier_chunk():
    """1023 nearby block ids plus one far outlier: the composite-key buckets
    are very uneven and the large ones take the warp sort."""
    n = 4096
    x = np.zeros(n, np.float32); y = np.zeros(n, np.float32); z = np.zeros(n, np.float32)
    for c in range(4):
        i = np.arange(1024, dtype=np.float32)
        x[c * 1024:(c + 1) * 1024] = i * 0.02 + c
        y[c * 1024:(c + 1) * 1024] = (i % 7) * 0.02
        x[c * 1024 + 517] = 1e4
    eb = 0.01
    seg, adj = po.seg_size(x, y, z, 3, 1, False, 0.0, eb)
    s_o = po.compress(x, y, z, 3, eb, seg)
    s_g, r = _gpu_compress(x, y, z, 3, eb, 1, "abs", 0.0)
    assert s_g == s_o
    _check_roundtrip(s_g, 3, 32)


def test_fallback_sort_sorted_input():
    """Spatially sorted points (heavy duplicates, narrow key ranges)."""
    x, y, z = po.generate(0, 50000, 3, 0.0, 10.0, 21, np.float32)
    order = np.lexsort((x, y, np.floor(z)))
    x, y, z = x[order].copy(), y[order].copy(), z[order].copy()
    for seg in (1, 32):
        s_o = po.compress(x, y, z, 3, 0.05, seg)
        s_g, r = _gpu_compress(x, y, z, 3, 0.05, seg, "abs", 0.0)
        assert s_g == s_o


def test_ranking_paths_mixed_within_warps():
    """Every warp encodes several chunks (5,860 chunks), and every third group of
    8 chunks is heavy: 300 points of each chunk in one small cube, the rest
    spread over the box.  The bucket ranking declines those chunks (a bucket
    of 16 or more points with 32-bit composites) to the warp sort, and the
    warp then ranks its next chunks by the warp sort directly before trying
    buckets again; the stream must equal the oracle's byte for byte."""
    n = 6_000_000
    rng = np.random.default_rng(77)
    x = (rng.random(n) * 1000.0).astype(np.float32)
    y = (rng.random(n) * 1000.0).astype(np.float32)
    z = (rng.random(n) * 1000.0).astype(np.float32)
    for c in range(0, n, 1024):
        if (c // 8192) % 3 != 0:
            continue
        m = min(300, n - c)
        sel = c + rng.choice(min(1024, n - c), m, replace=False)
        cx, cy, cz = rng.random(3) * 990.0
        x[sel] = (cx + rng.random(m) * 0.3).astype(np.float32)
        y[sel] = (cy + rng.random(m) * 0.3).astype(np.float32)
        z[sel] = (cz + rng.random(m) * 0.3).astype(np.float32)
    # segment 64: 157 blocks per axis, 32-bit composites of at least 21 bits
    eb = float(np.float32(0.05))
    s_o = po.compress(x, y, z, 3, eb, 64)
    s_g, r = _gpu_compress(x, y, z, 3, eb, 64, "abs", 0.0)
    assert r.status == 0 and s_g == s_o
    _check_roundtrip(s_g, 3, 32)


def test_float64_two_pass_decode_mixed_geometry():
    """Float64 chunks of ordinary geometry are decoded in the compact layout;
    chunks whose block-count product needs 64 bits are left to the general
    pass.  A stream with both kinds, chunk-aligned halves."""
    rng = np.random.default_rng(31)
    n, half = 40 * 1024, 20 * 1024
    axes = []
    for _ in range(3):
        a = np.empty(n, np.float64)
        a[:half] = rng.uniform(500.0, 500.05, half)   # about 250 blocks per axis
        a[half:] = rng.uniform(0.0, 1000.0, n - half)  # about 5e6 blocks per axis
        axes.append(a)
    run_arrays(axes[0], axes[1], axes[2], 3, 64, "abs", 1e-4, 1)
    # and the general pass alone: every chunk wide
    run_arrays(axes[0][half:].copy(), axes[1][half:].copy(), axes[2][half:].copy(), 3, 64, "abs", 1e-4, 1)


def test_unaligned_soa_views():
    """x, y, z carved from one buffer with n % 4 != 0 (the plugin layout,
    src/main.cpp:283-334): 4-byte aligned only, scalar path."""
    n = 10001
    x, y, z = po.generate(0, n, 3, 0.0, 50.0, 22, np.float32)
    buf = _t(np.concatenate([x, y, z]))
    tx, ty, tz = buf[:n], buf[n:2 * n], buf[2 * n:]
    assert ty.data_ptr() % 16 != 0
    s_g, r = gz.compress(tx, ty, tz, eb=0.01, seg_size=8)
    s_o = po.compress(x, y, z, 3, float(np.float32(0.01)), 8)
    assert s_g.cpu().numpy().tobytes() == s_o
    out = torch.zeros(3 * n + 1, dtype=torch.float32, device="cuda")
    ox, oy, oz = out[1:n + 1], out[n + 1:2 * n + 1], out[2 * n + 1:]
    scratch = torch.empty(256, dtype=torch.uint8, device="cuda")
    gz.decompress_into(s_g, s_g.numel(), 32, 3, ox, oy, oz, scratch)
    rx, ry, rz = po.decompress(s_o)
    assert np.array_equal(ox.cpu().numpy(), rx) and np.array_equal(oz.cpu().numpy(), rz)


def test_error_bound_per_point():
    """Every point within the bound (f32: within 1.01 eb for float rounding,
    the reference's own verification slack, src/utils.cu:28) via the
    oracle's permutation."""
    x, y, z = po.generate(1, 200000, 3, 0.0, 1000.0, 23, np.float32)
    eb = po.rel_to_abs(x, y, z, 1e-4)
    seg, _ = po.seg_size(x, y, z, 3, 0, True, float(np.float32(1e-4)), eb)
    s, r = gz.compress(_t(x), _t(y), _t(z), eb=eb, rel_mode=True, rel_eb=1e-4)
    assert r.id_overflow == 0
    dx, dy, dz = gz.decompress(s)
    perm = po.permutation(x, y, z, 3, eb, seg)
    for d, o in ((dx, x), (dy, y), (dz, z)):
        err = np.abs(d.cpu().numpy().astype(np.float64) - o[perm].astype(np.float64))
        assert err.max() <= 1.01 * eb


def test_safe31_keeps_bound_where_reference_masks():
    """The FCC f64 rel 1e-5 case overflows 31-bit block ids in the reference
    format (id_overflow); the SAFE31 extension doubles seg and holds the bound."""
    x, y, z = po.generate(2, 100000, 3, 0.0, 0.05, 24, np.float64)
    eb = po.rel_to_abs(x, y, z, 1e-5)
    s, r = gz.compress(_t(x), _t(y), _t(z), eb=eb, rel_mode=True, rel_eb=1e-5)
    assert r.id_overflow == 1
    s2, r2 = gz.compress(_t(x), _t(y), _t(z), eb=eb, rel_mode=True, rel_eb=1e-5, safe31=True)
    assert r2.status == 0 and r2.seg_size > r.seg_size and r2.adjusted == 1
    seg2, adj2 = po.seg_size(x, y, z, 3, 0, True, 1e-5, eb, True)
    assert seg2 == r2.seg_size
    assert s2.cpu().numpy().tobytes() == po.compress(x, y, z, 3, eb, seg2)
    dx, dy, dz = gz.decompress(s2)
    perm = po.permutation(x, y, z, 3, eb, seg2)
    for d, o in ((dx, x), (dy, y), (dz, z)):
        assert np.abs(d.cpu().numpy() - o[perm]).max() <= eb * (1 + 1e-9)


def test_seg_error_like_reference_exit():
    """Auto segment size > 1024 is the reference's exit(1) (src/cudaWarpCompress.cu:1547-1550);
    here GPZ_ESEG, as in the oracle."""
    x, y, z = po.generate(0, 5000, 3, 0.0, 1000.0, 25, np.float32)
    eb = float(np.float32(2.5e-4))
    with pytest.raises(po.OracleError) as eo:
        po.seg_size(x, y, z, 3, 1, False, 0.0, eb)
    assert eo.value.code == gz.GPZ_ESEG
    with pytest.raises(gz.GpzError) as ei:
        gz.compress(_t(x), _t(y), _t(z), eb=eb, seg_size=1)
    assert ei.value.code == gz.GPZ_ESEG


def test_rel_to_abs_matches_cli_host_arithmetic():
    for bits, dim in ((32, 3), (32, 2), (64, 3), (64, 2)):
        dt = np.float32 if bits == 32 else np.float64
        x, y, z = po.generate(1, 123457, dim, -20.0, 980.0, 26, dt)
        eb_o = po.rel_to_abs(x, y, z if dim == 3 else None, 1e-4)
        eb_g, mm = gz.rel_to_abs(_t(x), _t(y), _t(z) if dim == 3 else None, 1e-4)
        assert eb_g == eb_o


def test_scratch_reuse_and_streams():
    """Back-to-back calls on one scratch buffer and a side stream give identical bytes."""
    x, y, z = po.generate(0, 100000, 3, 0.0, 100.0, 27, np.float32)
    tx, ty, tz = _t(x), _t(y), _t(z)
    n = x.size
    p = gz.make_params(n, 3, 32, 0.01, 32)
    out = torch.empty(gz.stream_bound(n, 3, 32), dtype=torch.uint8, device="cuda")
    scratch = torch.empty(gz.compress_scratch_bytes(n), dtype=torch.uint8, device="cuda")
    ref = po.compress(x, y, z, 3, float(np.float32(0.01)), 32)
    side = torch.cuda.Stream()
    for st in (None, side, None):
        r = gz.compress_into(p, tx, ty, tz, out, scratch, stream=st)
        assert out[: r.stream_bytes].cpu().numpy().tobytes() == ref


def test_corrupted_streams_are_rejected_without_fault():
    x, y, z = po.generate(0, 30000, 3, 0.0, 100.0, 28, np.float32)
    s = bytearray(po.compress(x, y, z, 3, float(np.float32(0.01)), 32))
    G = (30000 + 1023) // 1024
    cases = {}
    t1 = bytes(s[: len(s) // 2])                      # truncated
    cases["truncated"] = t1
    t2 = bytearray(s); t2[24 + 8 * 3:24 + 8 * 3 + 8] = (10 ** 9).to_bytes(8, "little")  # offset past the end
    cases["offset"] = bytes(t2)
    t3 = bytearray(s); m = 24 + 8 * G + 36 * 2; t3[m + 34:m + 36] = (2000).to_bytes(2, "little")  # U > 1024
    cases["unique"] = bytes(t3)
    t4 = bytearray(s); t4[0:4] = (7).to_bytes(4, "little")  # dim
    cases["dim"] = bytes(t4)
    for name, blob in cases.items():
        d = _t(np.frombuffer(blob, np.uint8).copy())
        ox = torch.zeros(30000, device="cuda"); oy = torch.zeros_like(ox); oz = torch.zeros_like(ox)
        scratch = torch.empty(256, dtype=torch.uint8, device="cuda")
        with pytest.raises(gz.GpzError) as ei:
            gz.decompress_into(d, d.numel(), 32, 3, ox, oy, oz, scratch)
        assert ei.value.code == gz.GPZ_ESTREAM, name
    torch.cuda.synchronize()


def test_plugin_interface_mirror():
    """CompressorManager / CudaWarpCompress with the reference's buffer contract:
    input SoA in d_xyz is overwritten by the stream; the config's seg mutates."""
    n = 50000
    x, y, z = po.generate(0, n, 3, 0.0, 100.0, 29, np.float32)
    eb = po.rel_to_abs(x, y, z, 1e-4)
    cfg = gz.CudaConfig(seg_size=0, adjusted_seg=False, dim=3, coordinate_num=n, error_mode="rel",
                        eb=eb, rel_eb=float(np.float32(1e-4)), float_bits=32)
    comp = gz.CudaWarpCompress(cfg)
    mgr = gz.CompressorManager()
    d_xyz = _t(np.concatenate([x, y, z]))
    d_comp = torch.empty(4 * n * 4, dtype=torch.uint8, device="cuda")
    size = mgr.compressWarp(d_xyz, d_comp, "none", comp)
    seg, _ = po.seg_size(x, y, z, 3, 0, True, float(np.float32(1e-4)), eb)
    assert comp.getConfig().seg_size == seg
    s = d_xyz.view(torch.uint8)[:size].cpu().numpy().tobytes()
    assert s == po.compress(x, y, z, 3, eb, seg)
    h = mgr.decompressLoadParas("none", 0, 0, 0, s[:32])
    assert h == (3, n, 32)
    ox = torch.empty(n, device="cuda"); oy = torch.empty_like(ox); oz = torch.empty_like(ox)
    dec = gz.CudaWarpCompress()
    d_stream = torch.zeros(2 * n * 4, dtype=torch.uint8, device="cuda")
    d_stream[:size].copy_(d_xyz.view(torch.uint8)[:size])
    mgr.decompressWarp(ox, oy, oz, d_stream, dec, "none")
    rx, ry, rz = po.decompress(s)
    assert np.array_equal(ox.cpu().numpy(), rx) and np.array_equal(oz.cpu().numpy(), rz)
