"""The drop-in C++ surface: the `gpz` command line tool (same flags, messages and
prints as the reference's src/main.cpp:59-561) and the reference-compatible
classes of include/gpz/ (ICudaCompressor, CudaWarpCompress[Double],
CompressorManager, CudaConfig), which the tool drives.

CPU tests check argument validation (no CUDA call is reached) and that code
written against the reference headers compiles and links against the
library.  GPU tests run the tool end to end and compare with the reference
CLI's recorded output for the config-1 input (tests/golden/cases.json) and
with the oracle."""
import hashlib
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GPZ = os.path.join(ROOT, "gpz_b200", "gpz")
GOLDEN = os.path.join(ROOT, "tests", "golden", "cases.json")


def run(args, **kw):
    return subprocess.run([GPZ] + args, capture_output=True, text=True, timeout=600, **kw)


@pytest.fixture(scope="module", autouse=True)
def built():
    if not os.path.exists(GPZ):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "gpz_b200", "csrc")], check=True)


@pytest.mark.parametrize("args,msg", [
    ([], "Must specify either -x (compress) or -d (decompress)"),
    (["-x", "-d"], "Cannot specify both -x (compress) and -d (decompress)"),
    (["-x", "-i", "a", "-o", "b"], "Missing required arguments for compression"),
    (["-x", "-i", "a", "-o", "b", "-n", "10", "-m", "rel", "-e", "1e-4", "-f", "32", "-p", "4"],
     "Dimension must be 2 or 3"),
    (["-x", "-i", "a", "-o", "b", "-n", "10", "-m", "rel", "-e", "1e-4", "-f", "16"], "Float bits must be 32 or 64"),
    (["-x", "-i", "a", "-o", "b", "-n", "10", "-m", "rel", "-e", "1e-4", "-f", "32", "-t", "lz4"],
     "-t option requires nvcomp support"),
    (["-d", "-o", "b"], "-i and -o are required for decompression"),
])
def test_cli_argument_errors(args, msg):
    r = run(args)
    assert r.returncode == 1
    assert msg in r.stderr


def test_cli_missing_input_file(tmp_path):
    r = run(["-x", "-i", str(tmp_path / "nope.f32"), "-o", str(tmp_path / "o"), "-n", "10", "-m", "rel",
             "-e", "1e-4", "-f", "32"])
    assert r.returncode == 1 and "Failed to open input file" in r.stderr


def test_cli_input_size_checks(tmp_path):
    p = tmp_path / "in.f32"
    np.zeros(3 * 10 + 1, np.float32).tofile(p)
    r = run(["-x", "-i", str(p), "-o", str(tmp_path / "o"), "-n", "10", "-m", "rel", "-e", "1e-4", "-f", "32"])
    assert r.returncode == 1 and "not aligned to expected T struct" in r.stderr
    np.zeros(3 * 11, np.float32).tofile(p)
    r = run(["-x", "-i", str(p), "-o", str(tmp_path / "o"), "-n", "10", "-m", "rel", "-e", "1e-4", "-f", "32"])
    assert r.returncode == 1 and "does not match expected number of points" in r.stderr


def test_reference_headers_compile_and_link(tmp_path):
    """Code written against the reference's class declarations builds against
    include/gpz/ and links against libgpz_b200.so (no GPU call is made)."""
    src = tmp_path / "user.cpp"
    src.write_text(r'''
#include "CompressorManager.h"
#include <cstdio>
int main() {
  CudaConfig cfg(32, false, 3, 1000, "rel", 0.01f, 1e-4f, 32);
  CudaWarpCompress c(cfg);
  CudaWarpCompressDouble d(CudaConfig(16, false, 2, 500, "abs", 0.5, 0.0, 64));
  ICudaCompressor *i = &c;
  CompressorManager m;
  unsigned char hdr[24] = {3, 0, 0, 0, 0x40, 0x42, 0x0f, 0, 0, 0, 0, 0, 32, 0, 0, 0};
  uint32_t dim = 0, bits = 0; uint64_t n = 0;
  m.decompressLoadParas(&dim, &n, &bits, "none", 0, 0, 0, hdr);
  std::printf("%u %u %llu %u %u %u\n", i->getConfig().seg_size, d.getConfig().dim, (unsigned long long)n, dim, bits,
              ELEMS_PER_BLOCK);
  return 0;
}
''')
    exe = tmp_path / "user"
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include", "gpz"), "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", str(exe), "-L", os.path.join(ROOT, "gpz_b200"), "-lgpz_b200",
                    "-Wl,-rpath," + os.path.join(ROOT, "gpz_b200")], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    assert out == ["32", "2", "1000000", "3", "32", "1024"]


# ---------------------------------------------------------------------------- GPU

def _config1_input(tmp_path):
    from oracle import pyoracle as po
    x, y, z = po.generate(0, 1_000_000, 3, 0.0, 100.0, 1, np.float32)
    p = tmp_path / "cli_in.f32"
    np.stack([x, y, z], axis=1).astype(np.float32).tofile(p)
    return p, (x, y, z)


def _lines(text, prefixes):
    return [l for l in text.splitlines() if l.startswith(prefixes)]


@pytest.mark.gpu
def test_cli_compress_matches_reference_cli(tmp_path):
    """Config 1 through the CLI: the stream bytes and the deterministic printed
    lines equal the reference CLI's recorded run on the same file."""
    ref = json.load(open(GOLDEN))["cli_config1"]
    inp, _ = _config1_input(tmp_path)
    out = tmp_path / "cli_out.gpz"
    r = run(["-x", "-i", str(inp), "-o", str(out), "-n", "1000000", "-p", "3", "-f", "32", "-m", "rel", "-e", "1e-4"])
    assert r.returncode == 0, r.stderr
    data = out.read_bytes()
    assert len(data) == ref["bytes"]
    assert hashlib.sha256(data).hexdigest() == ref["stream_sha256"]
    assert data[:24].hex() == ref["header_hex"]
    keep = ("min_max_values", "Max Range", "Abs Error bound", "Segment size", "Adjusted Seg", "PCompression size",
            "PCompression ratio")
    assert _lines(r.stdout, keep) == _lines(ref["stdout"], keep)


@pytest.mark.gpu
def test_cli_round_trip_and_verify(tmp_path):
    """Compress then decompress through the CLI; the reconstruction equals the
    oracle's decode of the same stream and the reference-style verification
    counts no point off by more than 1.01*eb."""
    from oracle import pyoracle as po
    inp, (x, y, z) = _config1_input(tmp_path)
    stream = tmp_path / "s.gpz"
    r = run(["-x", "-i", str(inp), "-o", str(stream), "-n", "1000000", "-f", "32", "-m", "rel", "-e", "1e-4"])
    assert r.returncode == 0, r.stderr
    rec = tmp_path / "rec.f32"
    r = run(["-d", "-o", str(stream), "-r", str(rec), "-v", str(inp)])
    assert r.returncode == 0, r.stderr
    assert "Decompressed num points: 1000000" in r.stdout
    assert "Error Count: 0" in r.stdout
    got = np.fromfile(rec, np.float32).reshape(-1, 3)
    ox, oy, oz = po.decompress(stream.read_bytes())
    assert np.array_equal(got[:, 0].view(np.uint32), ox.view(np.uint32))
    assert np.array_equal(got[:, 1].view(np.uint32), oy.view(np.uint32))
    assert np.array_equal(got[:, 2].view(np.uint32), oz.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("bits,dim,mode,e,seg", [(64, 2, "rel", 1e-5, 0), (64, 3, "abs", 0.05, 8), (32, 2, "abs", 0.1, 4)])
def test_cli_streams_equal_oracle(tmp_path, bits, dim, mode, e, seg):
    """2D / f64 / abs-mode CLI runs: stream bytes equal the oracle's for the same
    absolute bound and segment size, and the decode equals the oracle's."""
    from oracle import pyoracle as po
    dt = np.float32 if bits == 32 else np.float64
    n = 70_001
    x, y, z = po.generate(1, n, dim, 0.0, 200.0, 11 + dim, dt)
    pts = np.stack([x, y] + ([z] if dim == 3 else []), axis=1).astype(dt)
    inp = tmp_path / "in.bin"
    pts.tofile(inp)
    stream = tmp_path / "s.gpz"
    args = ["-x", "-i", str(inp), "-o", str(stream), "-n", str(n), "-p", str(dim), "-f", str(bits), "-m", mode,
            "-e", repr(e)]
    if seg:
        args += ["-s", str(seg)]
    r = run(args)
    assert r.returncode == 0, r.stderr
    data = stream.read_bytes()
    h = po.parse_header(data)
    ref = po.compress(x, y, z, dim, h["eb"], h["seg"])
    assert data == bytes(ref)
    rec = tmp_path / "rec.bin"
    r = run(["-d", "-o", str(stream), "-r", str(rec)])
    assert r.returncode == 0, r.stderr
    got = np.fromfile(rec, dt).reshape(-1, dim)
    dec = po.decompress(data)
    for d in range(dim):
        assert np.array_equal(got[:, d], dec[d])
