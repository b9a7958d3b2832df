"""Generate the golden fixtures in tests/golden/ from the GPZ reference itself.

Runs the reference's own codec classes (CompressorManager + CudaWarpCompress /
CudaWarpCompressDouble), compiled from the reference sources by
``make -C oracle ref`` into ``oracle/_ref/``, on seeded synthetic inputs made
by the oracle's generators, and records:

* the compressed stream (full bytes for small cases, SHA-256 for all),
* the segment size / adjustment the reference chose,
* the reference's reconstruction (SHA-256, full bytes when small) for streams
  the reference decoder can run without its out-of-bounds write (no chunk
  with 1024 unique blocks; see oracle/ref_harness.cu),
* one run of the reference CLI (src/main.cpp) to pin the relative-bound
  conversion it performs on the host.

With ``--full`` it instead records, for the full-size workloads (FULL below:
the 143,735,721-point clustered float32 snapshot at rel 1e-4 and at abs 1e-3
with segment size 32, the 200,000,000-point float64 FCC lattice and the
100,000,000-point float64 2D square lattice at rel 1e-5), the SHA-256 of the
reference's stream and, where its decoder can run, of its reconstruction, in
``full_size.json``.

Needs a GPU:
    make -C oracle && make -C oracle ref    # once, where the reference sources are
    python tests/golden/make_golden.py --out <dir> [--full]
then copy <dir>/* into tests/golden/.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import pyoracle as po  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "gpz_ref_sm100a")
CLI = os.path.join(ROOT, "oracle", "_ref", "gpz")
FULL_BYTES_LIMIT = 160 * 1024

# name, kind, n, dim, bits, lo, hi, seed, mode, e, seg, special
CASES = [
    ("uni3d_f32_1m_rel1e-4", 0, 1_000_000, 3, 32, 0.0, 100.0, 1, "rel", 1e-4, 0, None),
    ("uni3d_f32_20k_rel1e-4", 0, 20_000, 3, 32, 0.0, 100.0, 2, "rel", 1e-4, 0, None),
    ("uni3d_f32_20481_rel1e-4", 0, 20_481, 3, 32, 0.0, 100.0, 3, "rel", 1e-4, 0, None),
    ("uni2d_f32_50k_rel1e-3", 0, 50_000, 2, 32, -50.0, 50.0, 4, "rel", 1e-3, 0, None),
    ("uni3d_f32_30k_rel1e-2", 0, 30_000, 3, 32, 0.0, 10.0, 5, "rel", 1e-2, 0, None),
    ("clu3d_f32_200k_abs1e-3_s32", 1, 200_000, 3, 32, 0.0, 1000.0, 6, "abs", 1e-3, 32, None),
    ("clu3d_f32_100k_rel1e-4", 1, 100_000, 3, 32, 0.0, 1000.0, 7, "rel", 1e-4, 0, None),
    ("clu3d_f32_60k_abs5e-1_s8", 1, 60_000, 3, 32, 0.0, 1000.0, 8, "abs", 0.5, 8, None),
    ("lat3d_f64_30k_rel1e-5", 2, 30_000, 3, 64, 0.0, 0.05, 9, "rel", 1e-5, 0, None),
    ("lat2d_f64_30k_rel1e-5", 2, 30_000, 2, 64, 0.0, 0.05, 10, "rel", 1e-5, 0, None),
    ("uni3d_f64_40k_rel1e-3", 0, 40_000, 3, 64, -1.0, 1.0, 11, "rel", 1e-3, 0, None),
    ("uni3d_f64_900k_rel1e-4", 0, 900_000, 3, 64, 0.0, 100.0, 12, "rel", 1e-4, 0, None),
    ("clu3d_f64_50k_abs2e-1_s16", 1, 50_000, 3, 64, 0.0, 1000.0, 13, "abs", 0.2, 16, None),
    ("signed_zero_f32", 0, 4096, 3, 32, 1.0, 2.0, 14, "abs", 1e-3, 4, "signed_zero"),
    ("signed_zero_f64", 0, 4096, 3, 64, 1.0, 2.0, 15, "abs", 1e-3, 4, "signed_zero"),
    ("const_f32", 0, 5000, 3, 32, 0.0, 1.0, 16, "abs", 1e-2, 2, "constant"),
    ("dups_f32", 0, 8192, 3, 32, 0.0, 4.0, 17, "abs", 1e-2, 16, "duplicates"),
    ("neg_f32_seg1", 0, 10_000, 3, 32, -300.0, -200.0, 18, "abs", 0.05, 1, None),
    ("wide_f32_seg512", 0, 12_000, 3, 32, 0.0, 1000.0, 19, "abs", 1e-3, 512, None),
    ("mask31_f32", 0, 20_000, 3, 32, 0.0, 1000.0, 22, "abs", 0.0104, 32, None),
    ("tail1_f32", 0, 3073, 3, 32, 0.0, 100.0, 20, "rel", 1e-4, 0, None),
    ("tail1023_f64_2d", 0, 4095, 2, 64, 0.0, 100.0, 21, "rel", 1e-4, 0, None),
]


# name, workload, n, dim, bits, mode, e, seg
FULL = [
    ("clustered_f32_143M_rel1e-4", "clustered", 143_735_721, 3, 32, "rel", 1e-4, 0),
    ("clustered_f32_143M_abs1e-3_s32", "clustered", 143_735_721, 3, 32, "abs", 1e-3, 32),
    ("fcc_f64_200M_rel1e-5", "fcc", 200_000_000, 3, 64, "rel", 1e-5, 0),
    ("square_f64_100M_rel1e-5", "square", 100_000_000, 2, 64, "rel", 1e-5, 0),
]


def full_input(workload, n):
    """Host SoA arrays (x, y, z) of a full-size workload; z is zeros in 2D.

    clustered: the bench generator (70 % in 20,000 Gaussian clusters, 30 %
    uniform, box [0,1000)^3, shuffled; seed 1234), drawn on cuda:0.
    fcc / square: the oracle's lattice generator (spacing 1, Gaussian jitter
    sigma 0.05, random order; seed 2024)."""
    if workload == "clustered":
        import bench
        return tuple(t.cpu().numpy() for t in bench.gen_clustered(n, 1234, "cuda"))
    dim = 3 if workload == "fcc" else 2
    return po.generate(2, n, dim, 0.0, 0.05, 2024, np.float64)


def full_eb(x, y, z, dim, bits, mode, e):
    """The absolute bound the reference CLI passes to the codec."""
    if mode != "rel":
        return float(np.float32(e)) if bits == 32 else float(e)
    return po.rel_to_abs(x, y, z if dim == 3 else None, e)


def sha_array(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(memoryview(np.ascontiguousarray(a)).cast("B"))
    return h.hexdigest()


def main_full(args):
    tmp = tempfile.mkdtemp(prefix="gpz_golden_full_")
    recs = []
    for (name, workload, n, dim, bits, mode, e, seg) in FULL:
        x, y, z = full_input(workload, n)
        eb = full_eb(x, y, z, dim, bits, mode, e)
        soa = os.path.join(tmp, "in.soa")
        with open(soa, "wb") as f:
            for a in (x, y, z):
                f.write(memoryview(np.ascontiguousarray(a)).cast("B"))
        del x, y, z
        sfile = os.path.join(tmp, "out.gpz")
        rc, out, err = run([HARNESS, "compress", soa, str(n), str(dim), str(bits), repr(eb), repr(e), mode,
                            str(seg), sfile, "1"])
        os.remove(soa)
        rec = dict(name=name, workload=workload, n=n, dim=dim, bits=bits, mode=mode, e=e, seg_in=seg, eb=eb)
        if rc != 0:
            rec["compress_error"] = (out + err).strip()[-400:]
            recs.append(rec)
            print(name, "compress failed", rc, err[-300:], flush=True)
            continue
        info = json.loads(out.strip().splitlines()[-1])
        stream = np.fromfile(sfile, np.uint8)
        rec.update(seg=info["seg"], adjusted=info["adjusted"], bytes=int(stream.size),
                   stream_sha256=sha_array(stream), compress_ms=info["ms"])
        del stream
        dfile = os.path.join(tmp, "out.dec")
        rc, out, err = run([HARNESS, "decompress", sfile, dfile, "1"])
        if rc == 0:
            dec = np.fromfile(dfile, np.uint8)
            # the harness writes three axes; a 2D stream's third is zeros
            rec["decoded_sha256"] = sha_array(dec[: dim * n * bits // 8])
            rec["decompress_ms"] = json.loads(out.strip().splitlines()[-1])["ms"]
            del dec
            os.remove(dfile)
        elif rc == 3:
            rec["decompress_refused"] = out.strip()
        else:
            rec["decompress_error"] = (out + err).strip()[-400:]
        os.remove(sfile)
        recs.append(rec)
        print(json.dumps(rec), flush=True)
    with open(os.path.join(args.out, "full_size.json"), "w") as f:
        json.dump(dict(fixtures=recs), f, indent=1)
    shutil.rmtree(tmp, ignore_errors=True)


def make_input(kind, n, dim, bits, lo, hi, seed, special):
    dtype = np.float32 if bits == 32 else np.float64
    x, y, z = po.generate(kind, n, dim, lo, hi, seed, dtype)
    if special == "signed_zero":
        # chunk 0: x min is -0.0 at lane 5 and +0.0 at lane 700; chunk 1 swaps
        # them; chunk 2: y max candidates -0.0 / +0.0 with every other y < 0.
        x[5], x[700] = -0.0, 0.0
        x[1024 + 5], x[1024 + 700] = 0.0, -0.0
        y[2048:3072] = -y[2048:3072]
        y[2048 + 3], y[2048 + 900] = -0.0, 0.0
        y[3072:4096] = -y[3072:4096]
        y[3072 + 3], y[3072 + 900] = 0.0, -0.0
    elif special == "constant":
        x[:] = dtype(0.25); y[:] = dtype(-3.5); z[:] = dtype(7.0)
    elif special == "duplicates":
        q = np.round(x * 4) / 4
        x[:] = q; y[:] = np.round(y * 4) / 4; z[:] = np.round(z * 4) / 4
    if dim == 2:
        z[:] = 0
    return x, y, z


def sha(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def run(cmd):
    p = subprocess.run(cmd, capture_output=True, text=True)
    return p.returncode, p.stdout, p.stderr


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--full", action="store_true", help="record the full-size workloads (full_size.json)")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    if args.full:
        main_full(args)
        return
    tmp = tempfile.mkdtemp(prefix="gpz_golden_")
    fixtures = []
    for (name, kind, n, dim, bits, lo, hi, seed, mode, e, seg, special) in CASES:
        x, y, z = make_input(kind, n, dim, bits, lo, hi, seed, special)
        if mode == "rel":
            eb = po.rel_to_abs(x, y, z if dim == 3 else None, e)
        else:
            eb = e
        soa = os.path.join(tmp, name + ".soa")
        np.concatenate([x, y, z]).tofile(soa)
        sfile = os.path.join(tmp, name + ".gpz")
        rc, out, err = run([HARNESS, "compress", soa, str(n), str(dim), str(bits), repr(eb), repr(e),
                            mode, str(seg), sfile, str(args.reps)])
        rec = dict(name=name, kind=kind, n=n, dim=dim, bits=bits, lo=lo, hi=hi, seed=seed, mode=mode,
                   e=e, seg_in=seg, special=special, eb=eb)
        if rc != 0:
            rec["compress_error"] = (out + err).strip()[-400:]
            fixtures.append(rec)
            print(name, "compress failed", rc, err[-300:], flush=True)
            continue
        info = json.loads(out.strip().splitlines()[-1])
        stream = open(sfile, "rb").read()
        rec.update(seg=info["seg"], adjusted=info["adjusted"], bytes=len(stream), stream_sha256=sha(stream),
                   compress_ms=info["ms"])
        if len(stream) <= FULL_BYTES_LIMIT:
            with open(os.path.join(args.out, name + ".gpz"), "wb") as f:
                f.write(stream)
            rec["stream_file"] = name + ".gpz"
        dfile = os.path.join(tmp, name + ".dec")
        rc, out, err = run([HARNESS, "decompress", sfile, dfile, str(args.reps)])
        if rc == 0:
            dec = open(dfile, "rb").read()
            rec["decoded_sha256"] = sha(dec)
            rec["decompress_ms"] = json.loads(out.strip().splitlines()[-1])["ms"]
            if len(dec) <= FULL_BYTES_LIMIT:
                with open(os.path.join(args.out, name + ".dec"), "wb") as f:
                    f.write(dec)
                rec["decoded_file"] = name + ".dec"
        elif rc == 3:
            rec["decompress_refused"] = out.strip()
        else:
            rec["decompress_error"] = (out + err).strip()[-400:]
        fixtures.append(rec)
        print(name, {k: rec.get(k) for k in ("seg", "adjusted", "bytes")}, flush=True)

    # The reference CLI on config-1-sized input: pins the host-side rel->abs
    # conversion (the stream header carries the absolute bound at byte 16).
    x, y, z = make_input(0, 1_000_000, 3, 32, 0.0, 100.0, 1, None)
    aos = os.path.join(tmp, "cli_in.f32")
    np.stack([x, y, z], axis=1).astype(np.float32).tofile(aos)
    cli_out = os.path.join(tmp, "cli_out.gpz")
    rc, out, err = run([CLI, "-x", "-i", aos, "-o", cli_out, "-n", "1000000", "-p", "3", "-f", "32",
                        "-m", "rel", "-e", "1e-4"])
    cli = dict(returncode=rc, stdout=out[-2000:])
    if rc == 0:
        s = open(cli_out, "rb").read()
        cli.update(bytes=len(s), stream_sha256=sha(s), header_hex=s[:24].hex())
    with open(os.path.join(args.out, "cases.json"), "w") as f:
        json.dump(dict(fixtures=fixtures, cli_config1=cli), f, indent=1)
    shutil.rmtree(tmp, ignore_errors=True)
    print("done", len(fixtures))


if __name__ == "__main__":
    main()
