"""Times the GPZ reference's own GPU codec on the bench workloads and checks
this repository's codec against it.

TEST INFRASTRUCTURE ONLY: a measurement recipe beside the reference build of
oracle/Makefile (target `ref`), not part of the product.  For a workload it
1. generates the points and computes the absolute bound as the reference CLI
   does (convertRelEb on the per-axis ranges) or takes the given one;
2. compresses and decompresses them with this repository's codec (CUDA-event
   times, mean of the repetitions after one warm-up) and checks every point
   with gpz_verify, also in the GPZ_FLAG_SAFE31 mode;
3. writes them as SoA to a temporary file and runs the reference harness
   (oracle/_ref/gpz_ref_sm100a and, with --ptx90, the stock compute_90 PTX
   build) through the reference's CompressorManager;
4. prints one JSON line per build: times, GB/s of input bytes, and whether
   the reference's stream and reconstruction are identical to this codec's.

Workloads:
  clustered  143,735,721 float32 3D points, the bench generator (seed 1234), rel 1e-4
             (--mode abs --eb 1e-3 --seg 32 for the absolute-bound run)
  fcc        200,000,000 float64 3D points, FCC lattice (369^3 cells truncated),
             jitter sigma 0.05, random order, rel 1e-5
  square     100,000,000 float64 2D points, square lattice, same jitter, rel 1e-5

    python oracle/time_reference_gpu.py [--workload W] [--reps R] [--ptx90]
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def points(workload, n):
    import numpy as np
    import torch
    if workload == "clustered":
        import bench
        return bench.gen_clustered(n, 1234, "cuda"), 32, 3
    from oracle import pyoracle as po
    dim = 3 if workload == "fcc" else 2
    x, y, z = po.generate(2, n, dim, 0.0, 0.05, 2024, np.float64)
    t = [torch.from_numpy(a).cuda() for a in (x, y, z)]
    return (t[0], t[1], t[2] if dim == 3 else None), 64, dim


def event_ms(fn, reps):
    import torch
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", choices=["clustered", "fcc", "square"], default="clustered")
    ap.add_argument("--points", type=int, default=0)
    ap.add_argument("--mode", choices=["rel", "abs"], default="rel")
    ap.add_argument("--eb", type=float, default=0.0, help="relative bound (rel mode; 0 = workload default) or absolute")
    ap.add_argument("--seg", type=int, default=0, help="segment size (abs mode needs one)")
    ap.add_argument("--reps", type=int, default=4)
    ap.add_argument("--ptx90", action="store_true")
    ap.add_argument("--tmp", default=tempfile.gettempdir())
    args = ap.parse_args()
    import numpy as np
    import torch
    import gpz_b200 as gz
    n = args.points or {"clustered": 143_735_721, "fcc": 200_000_000, "square": 100_000_000}[args.workload]
    (x, y, z), bits, dim = points(args.workload, n)
    dt = np.float32 if bits == 32 else np.float64
    rel_mode = args.mode == "rel"
    rel = (args.eb or (1e-4 if args.workload == "clustered" else 1e-5)) if rel_mode else 0.0
    if rel_mode:
        rng = [dt(a.max().item()) - dt(a.min().item()) for a in (x, y, z) if a is not None]
        eb = dt(max(rng + [dt(0)])) * dt(rel)
    else:
        eb = dt(args.eb)
    rel_arg = float(dt(rel)) if rel_mode else 0.0
    # ---- this codec: timing and verification
    s, res = gz.compress(x, y, z, eb=float(eb), seg_size=args.seg, rel_mode=rel_mode, rel_eb=rel_arg)
    p = gz.make_params(n, dim, bits, float(eb), args.seg, rel_mode, rel_arg)
    cap = gz.stream_bound(n, dim, bits)
    out = torch.empty(cap, dtype=torch.uint8, device="cuda")
    scr = torch.empty(gz.compress_scratch_bytes(n), dtype=torch.uint8, device="cuda")
    c_ms = event_ms(lambda: gz.compress_into(p, x, y, z if z is not None else x, out, scr, sync=False), args.reps)
    dx, dy, dz = gz.decompress(s)
    sd = torch.empty(256, dtype=torch.uint8, device="cuda")
    d_ms = event_ms(lambda: gz.decompress_into(s, s.numel(), bits, dim, dx, dy, dz if dim == 3 else dx, sd, sync=False),
                    args.reps)
    v = gz.verify(x, y, z, dx, dy, dz, float(eb), res.seg_size)
    p31 = gz.make_params(n, dim, bits, float(eb), args.seg, rel_mode, rel_arg, safe31=True)
    r31 = gz.compress_into(p31, x, y, z if z is not None else x, out, scr)
    s31 = out[: r31.stream_bytes].clone()
    ex, ey, ez = gz.decompress(s31)
    v31 = gz.verify(x, y, z, ex, ey, ez, float(eb), r31.seg_size)
    inb = dim * n * bits // 8
    ours = {"workload": args.workload, "points": n, "bits": bits, "dim": dim, "mode": args.mode, "eb": float(eb),
            "seg": int(res.seg_size), "stream_bytes": int(res.stream_bytes), "id_overflow": int(res.id_overflow),
            "compress_ms": round(c_ms, 3), "compress_gbs": round(inb / c_ms / 1e6, 2),
            "decompress_ms": round(d_ms, 3), "decompress_gbs": round(inb / d_ms / 1e6, 2),
            "over_1.01eb": int(v.over_bound_tol), "psnr_db": round(v.psnr_combined, 3),
            "safe31": {"seg": int(r31.seg_size), "stream_bytes": int(r31.stream_bytes),
                       "over_1.01eb": int(v31.over_bound_tol)}}
    print(json.dumps({"build": "gpz_b200", **ours}), flush=True)
    ours_h = s.cpu().numpy()
    ours_rec = torch.cat([t for t in (dx, dy, dz) if t is not None]).cpu().numpy().view(np.uint8)
    soa = os.path.join(args.tmp, "gpz_ref_in.soa")
    with open(soa, "wb") as f:  # the harness reads three axes; 2D data has z = 0, as the reference loader sets it
        for a in (x, y, z):
            f.write(a.cpu().numpy().tobytes() if a is not None else bytes(n * bits // 8))
    del x, y, z, s, dx, dy, dz, ex, ey, ez, out, s31
    torch.cuda.empty_cache()
    # ---- the reference
    builds = ["gpz_ref_sm100a"] + (["gpz_ref_ptx90"] if args.ptx90 else [])
    for b in builds:
        exe = os.path.join(ROOT, "oracle", "_ref", b)
        st = os.path.join(args.tmp, b + ".gpz")
        rc = subprocess.run([exe, "compress", soa, str(n), str(dim), str(bits), repr(float(eb)), repr(rel), args.mode,
                             str(args.seg), st, str(args.reps)], capture_output=True, text=True)
        if rc.returncode != 0:
            print(json.dumps({"build": b, "op": "compress", "error": rc.stderr.strip()[-300:]}))
            continue
        c = json.loads(rc.stdout.strip().splitlines()[-1])
        rec = os.path.join(args.tmp, b + ".rec")
        rd = subprocess.run([exe, "decompress", st, rec, str(args.reps)], capture_output=True, text=True)
        d = json.loads(rd.stdout.strip().splitlines()[-1]) if rd.returncode in (0, 3) and rd.stdout.strip() else {
            "error": rd.stderr.strip()[-300:]}
        cms = min(c["ms"][1:] or c["ms"])
        outl = {"build": b, "points": n, "eb": float(eb), "seg": c["seg"], "stream_bytes": c["bytes"],
                "compress_ms": c["ms"], "compress_gbs_best": round(inb / cms / 1e6, 2)}
        if "ms" in d:
            dms = min(d["ms"][1:] or d["ms"])
            outl.update(decompress_ms=d["ms"], decompress_gbs_best=round(inb / dms / 1e6, 2))
        else:
            outl.update(decompress=d)
        ref_stream = np.fromfile(st, np.uint8)
        outl["stream_identical_to_gpz_b200"] = bool(ref_stream.size == ours_h.size and np.array_equal(ref_stream, ours_h))
        if os.path.exists(rec) and "ms" in d:
            # the harness writes three axes; a 2D stream's third is zeros
            outl["reconstruction_identical_to_gpz_b200"] = bool(
                np.array_equal(np.fromfile(rec, np.uint8)[: ours_rec.size], ours_rec))
        print(json.dumps(outl), flush=True)
        for q in (st, rec):
            if os.path.exists(q):
                os.remove(q)
    os.remove(soa)


if __name__ == "__main__":
    main()
