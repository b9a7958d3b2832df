"""Times the GPZ reference's own GPU codec on the bench workload.

TEST INFRASTRUCTURE ONLY: a measurement recipe beside the reference build of
oracle/Makefile (target `ref`), not part of the product.  It generates the
bench's clustered float32 3D snapshot (bench.gen_clustered, same seed), writes
it as SoA to a temporary file, runs the reference harness
(oracle/_ref/gpz_ref_sm100a and, with --ptx90, the stock compute_90 PTX build)
for compress and decompress through the reference's CompressorManager, and
prints one JSON line per build with the CUDA-event times and GB/s of input
bytes.  It also compresses and decompresses the same data with this
repository's codec and reports whether the stream bytes and the
reconstruction are identical to the reference's.  The same data through this
repository's codec is timed by bench.py.

    python oracle/time_reference_gpu.py [--points N] [--reps R] [--ptx90]
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--points", type=int, default=143_735_721)
    ap.add_argument("--reps", type=int, default=4)
    ap.add_argument("--ptx90", action="store_true")
    ap.add_argument("--tmp", default=tempfile.gettempdir())
    args = ap.parse_args()
    import numpy as np
    import torch
    import bench
    x, y, z = bench.gen_clustered(args.points, 1234, "cuda")
    rel = 1e-4
    # the harness takes the absolute bound: convertRelEb<float> of the CLI
    # (src/main.cpp:35-55) on the per-axis float ranges
    rng = [np.float32(a.max().item()) - np.float32(a.min().item()) for a in (x, y, z)]
    eb = np.float32(max(rng)) * np.float32(rel)
    soa = os.path.join(args.tmp, "gpz_ref_in.soa")
    with open(soa, "wb") as f:
        for a in (x, y, z):
            f.write(a.cpu().numpy().tobytes())
    inb = 3 * 4 * args.points
    import gpz_b200 as gz
    ours, res = gz.compress(x, y, z, eb=float(eb), rel_mode=True, rel_eb=float(np.float32(rel)))
    ours_h = ours.cpu().numpy()
    dx, dy, dz = gz.decompress(ours)
    ours_rec = torch.cat([dx, dy, dz]).cpu().numpy().view(np.uint32)
    del x, y, z, ours, dx, dy, dz
    torch.cuda.empty_cache()
    builds = ["gpz_ref_sm100a"] + (["gpz_ref_ptx90"] if args.ptx90 else [])
    for b in builds:
        exe = os.path.join(ROOT, "oracle", "_ref", b)
        st = os.path.join(args.tmp, b + ".gpz")
        rc = subprocess.run([exe, "compress", soa, str(args.points), "3", "32", repr(float(eb)), str(rel), "rel", "0", st,
                             str(args.reps)], capture_output=True, text=True)
        if rc.returncode != 0:
            print(json.dumps({"build": b, "op": "compress", "error": rc.stderr.strip()[-300:]}))
            continue
        c = json.loads(rc.stdout.strip().splitlines()[-1])
        rec = os.path.join(args.tmp, b + ".rec")
        rd = subprocess.run([exe, "decompress", st, rec, str(args.reps)], capture_output=True, text=True)
        d = json.loads(rd.stdout.strip().splitlines()[-1]) if rd.returncode in (0, 3) and rd.stdout.strip() else {
            "error": rd.stderr.strip()[-300:]}
        cms = min(c["ms"][1:] or c["ms"])
        out = {"build": b, "points": args.points, "eb": float(eb), "seg": c["seg"], "stream_bytes": c["bytes"],
               "compress_ms": c["ms"], "compress_gbs_best": round(inb / cms / 1e6, 2)}
        if "ms" in d:
            dms = min(d["ms"][1:] or d["ms"])
            out.update(decompress_ms=d["ms"], decompress_gbs_best=round(inb / dms / 1e6, 2))
        else:
            out.update(decompress=d)
        ref_stream = np.fromfile(st, np.uint8)
        out["stream_identical_to_gpz_b200"] = bool(ref_stream.size == ours_h.size and np.array_equal(ref_stream, ours_h))
        if os.path.exists(rec) and "ms" in d:
            out["reconstruction_identical_to_gpz_b200"] = bool(np.array_equal(np.fromfile(rec, np.uint32), ours_rec))
        print(json.dumps(out))
        for p in (st, rec):
            if os.path.exists(p):
                os.remove(p)
    os.remove(soa)


if __name__ == "__main__":
    main()
