"""Benchmark: compress + decompress of the 143,735,721-point float32 3D particle
snapshot (70 % in 20,000 Gaussian clusters with Pareto(1.5) populations, 30 %
uniform background, box [0,1000)^3, shuffled; relative error bound 1e-4,
automatic segment size) on B200 GPUs.

One step = one compress of the snapshot followed by one decompress of the
resulting stream.  `value` is the uncompressed input bytes (N * 3 * 4 per rank,
summed over ranks) divided by the step time (compress + decompress), in GB/s
(1e9), with the inputs resident in HBM.  `e2e` is the same metric through the
C ABI with pinned host buffers: every step copies the SoA input to the device,
compresses, reads the stream back, copies it to the device again, decompresses
and reads the reconstruction back.

Multi-GPU: one process per GPU (torchrun); every rank compresses its own
snapshot (seed + rank), so the work per GPU is fixed (weak scaling) and no
collective touches the data path.  Time is the max over ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`--impl reference` times the CPU implementation of the same path on the box's
host cores: the project's OpenMP restatement of the reference algorithm
(oracle/), since the reference itself only has a GPU implementation.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_POINTS = 143_735_721
REL_EB = 1e-4
WORKLOAD = ("143,735,721 float32 3D points, 70% in 20,000 Gaussian clusters (sigma log-uniform "
            "[0.5,10], Pareto(1.5) populations) + 30% uniform, box [0,1000)^3, shuffled; "
            "rel error bound 1e-4, automatic segment size")
METRIC = "compress & decompress GB/s (input bytes) on 1 B200, % of HBM roofline; batched vs plain"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_from_profile(n, kernel):
    """DRAM bytes per launch of the compress / decompress kernel on the default
    143.7M-point workload, from the committed ncu summary (None otherwise)."""
    p = os.path.join(ROOT, "profiles", f"{kernel}_kernel_143M_f32_3d.md")
    if n != N_POINTS or not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def bench_config(w, n, world, seg, sbytes):
    """The `config` object of the JSON line (both arms print the same keys)."""
    inb = n * w["dim"] * w["bits"] // 8
    return {"workload": w["desc"], "points_per_gpu": n, "dim": w["dim"], "float_bits": w["bits"],
            "error_mode": w["mode"], "error_bound": w["e"], "segment_size_requested": w["seg"],
            "segment_size": int(seg), "stream_bytes": int(sbytes), "compression_ratio": round(inb / sbytes, 4),
            "parallelism": f"{world} independent snapshots",
            "l2": f"inputs ({inb / 1e9:.2f} GB per GPU) larger than the 126 MB L2; no flush"}


def gen_clustered(n, seed, device):
    """Synthetic stand-in for the SDRBench/HACC-style snapshot (not in this container)."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    K = 20000
    cen = torch.rand(K, 3, generator=g, device=device) * 1000
    sig = 0.5 * 20 ** torch.rand(K, generator=g, device=device)
    w = (1 - torch.rand(K, generator=g, device=device)) ** (-1 / 1.5)
    cdf = torch.cumsum(w.double(), 0)
    ncl = int(0.7 * n)
    u = torch.rand(ncl, generator=g, device=device, dtype=torch.float64) * cdf[-1]
    idx = torch.searchsorted(cdf, u).clamp_(max=K - 1)
    p = torch.empty(n, 3, device=device)
    p[:ncl] = (cen[idx] + sig[idx, None] * torch.randn(ncl, 3, generator=g, device=device)).clamp_(0, 999.999)
    p[ncl:] = torch.rand(n - ncl, 3, generator=g, device=device) * 1000
    p = p[torch.randperm(n, generator=g, device=device)]
    out = [p[:, d].contiguous() for d in range(3)]
    del p, idx, u
    return out


def gen_lattice(n, dim, seed, device):
    """Jittered lattice snapshot, float64, shuffled: FCC (3D; 4 points per
    cubic cell of edge 1, 369^3 cells truncated to n) or square (2D; side
    10,000, spacing 1), Gaussian thermal displacement sigma 0.05 per axis."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    i = torch.arange(n, device=device, dtype=torch.int64)
    if dim == 3:
        cells = 369
        cell, b = i // 4, i % 4
        del i
        basis = torch.tensor([[0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]],
                             dtype=torch.float64, device=device)
        out = []
        for d, c in enumerate((cell % cells, (cell // cells) % cells, cell // (cells * cells))):
            out.append(c.double() + basis[b, d])
        del cell, b
    else:
        side = 10_000
        out = [(i % side).double(), (i // side).double()]
        del i
    perm = torch.randperm(n, generator=g, device=device)
    res = []
    for a in out:
        a += 0.05 * torch.randn(n, generator=g, device=device, dtype=torch.float64)
        res.append(a[perm].contiguous())
    del out, perm
    return res + ([None] if dim == 2 else [])


# name -> workload (the default, "clustered", is the headline)
WORKLOADS = {
    "clustered": dict(n=N_POINTS, dim=3, bits=32, mode="rel", e=REL_EB, seg=0, gen="clustered", desc=WORKLOAD),
    "clustered-abs": dict(n=N_POINTS, dim=3, bits=32, mode="abs", e=1e-3, seg=32, gen="clustered",
                          desc=WORKLOAD.replace("rel error bound 1e-4, automatic segment size",
                                                "abs error bound 1e-3, segment size 32 (raised to 512 by the "
                                                "reference's block-count rule)")),
    "fcc": dict(n=200_000_000, dim=3, bits=64, mode="rel", e=1e-5, seg=0, gen="lattice",
                desc="200,000,000 float64 3D points of an FCC lattice (edge 1, 369^3 cells truncated), Gaussian "
                     "jitter sigma 0.05, shuffled; rel error bound 1e-5, automatic segment size"),
    "square": dict(n=100_000_000, dim=2, bits=64, mode="rel", e=1e-5, seg=0, gen="lattice",
                   desc="100,000,000 float64 2D points of a square lattice (side 10,000, spacing 1), Gaussian "
                        "jitter sigma 0.05, shuffled; rel error bound 1e-5, automatic segment size"),
}


def gen_workload(w, n, seed, device):
    if w["gen"] == "clustered":
        return gen_clustered(n, seed, device)
    return gen_lattice(n, w["dim"], seed, device)


def typed(bits, v):
    import numpy as np
    return float(np.float32(v)) if bits == 32 else float(v)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(prefix="gpz_clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n_gpus):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    import torch
    if torch.cuda.is_available():
        torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    if torch.cuda.is_available():
        torch.cuda.synchronize()


def cpu_baseline_run(w, x, y, z, steps=1):
    """Times the OpenMP oracle (compress + decompress) on all host cores."""
    import numpy as np
    from oracle import pyoracle as po
    cores = os.cpu_count() or 1
    dim, bits = w["dim"], w["bits"]
    if z is None:
        z = np.zeros_like(x)
    rel_mode = w["mode"] == "rel"
    eb = typed(bits, po.rel_to_abs(x, y, z if dim == 3 else None, w["e"]) if rel_mode else w["e"])
    seg, _ = po.seg_size(x, y, z, dim, w["seg"], rel_mode, typed(bits, w["e"]), eb)
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        s = po.compress(x, y, z, dim, eb, seg, nthreads=cores)
        po.decompress(s, nthreads=cores)
        ts.append(time.perf_counter() - t0)
    return ts, cores, len(s), seg


REF_BUILDS = (("gpz_ref_sm100a", "reference sources built for sm_100a"),
              ("gpz_ref_ptx90", "stock CMake architectures (compute_90 PTX, JIT-compiled on the B200)"))


def reference_gpu_run(w, hx, hy, hz, n, eb, rel, ours_stream, ours_rec, reps):
    """Times the reference's own GPU codec on the same snapshot, in this run.

    The reference is built from its sources by oracle/Makefile (target `ref`)
    into oracle/_ref/; its harness (oracle/ref_harness.cu) drives the
    reference's CompressorManager with the CLI's scratch and buffer sizes and
    times compressWarp / decompressWarp with CUDA events, the scope of the
    reference CLI's own timer (src/main.cpp:336-346).  The first repetition
    (PTX JIT, first-touch) is dropped.  Its stream and reconstruction are
    compared byte for byte with this codec's."""
    import numpy as np
    out = {}
    exes = {b: os.path.join(ROOT, "oracle", "_ref", b) for b, _ in REF_BUILDS}
    if not any(os.path.exists(e) for e in exes.values()):
        return {"unavailable": "reference build oracle/_ref/ not present (make -C oracle ref)"}
    tmp = tempfile.mkdtemp(prefix="gpz_refgpu_")
    soa = os.path.join(tmp, "in.soa")
    dim, bits = w["dim"], w["bits"]
    with open(soa, "wb") as f:  # the harness reads three axes; a 2D snapshot's third is zeros
        for a in (hx, hy, hz):
            f.write(memoryview(a.numpy()).cast("B") if a is not None else bytes(n * bits // 8))
    inb = n * dim * bits // 8
    try:
        for b, what in REF_BUILDS:
            exe = exes[b]
            if not os.path.exists(exe):
                out[b] = {"unavailable": "not built"}
                continue
            st, rec = os.path.join(tmp, "ref.gpz"), os.path.join(tmp, "ref.rec")
            p = subprocess.run([exe, "compress", soa, str(n), str(dim), str(bits), repr(eb), repr(rel), w["mode"],
                                str(w["seg"]), st, str(reps + 1)], capture_output=True, text=True)
            if p.returncode != 0:
                out[b] = {"unavailable": "compress failed: " + (p.stdout + p.stderr).strip()[-200:]}
                continue
            c = json.loads(p.stdout.strip().splitlines()[-1])
            cms = c["ms"][1:] or c["ms"]
            d = subprocess.run([exe, "decompress", st, rec, str(reps + 1)], capture_output=True, text=True)
            rs = np.fromfile(st, np.uint8)
            line = {"build": what, "compress_ms_best": round(min(cms), 4),
                    "compress_ms_median": round(statistics.median(cms), 4),
                    "compress_gbs_best": round(inb / min(cms) / 1e6, 2), "stream_bytes": int(c["bytes"]),
                    "segment_size": int(c["seg"]),
                    "identical_stream": bool(rs.size == ours_stream.size and np.array_equal(rs, ours_stream))}
            del rs
            if d.returncode == 0:
                dj = json.loads(d.stdout.strip().splitlines()[-1])
                dms = dj["ms"][1:] or dj["ms"]
                rr = np.fromfile(rec, np.uint8)[: ours_rec.size]  # the harness writes three axes
                line.update(decompress_ms_best=round(min(dms), 4), decompress_ms_median=round(statistics.median(dms), 4),
                            decompress_gbs_best=round(inb / min(dms) / 1e6, 2),
                            identical_reconstruction=bool(rr.size == ours_rec.size and np.array_equal(rr, ours_rec)))
                del rr
            else:
                line["decompress"] = "not run: " + (d.stdout + d.stderr).strip()[-200:]
            line["reps"] = len(cms)
            out[b] = line
            for q in (st, rec):
                if os.path.exists(q):
                    os.remove(q)
    finally:
        if os.path.exists(soa):
            os.remove(soa)
        os.rmdir(tmp)
    return out


def run_reference(args):
    """CPU implementation of the path on the host cores (rank 0 only)."""
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = WORKLOADS[args.config]
    n = args.points or w["n"]
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    axes = gen_workload(w, n, 1234 if w["gen"] == "clustered" else 2024, dev)
    x, y = (t.cpu().numpy() for t in axes[:2])
    z = axes[2].cpu().numpy() if axes[2] is not None else None
    del axes
    if args.warmup > 0:
        cpu_baseline_run(w, x, y, z, args.warmup)
    ts, cores, sbytes, seg = cpu_baseline_run(w, x, y, z, args.steps)
    step = sum(ts) / len(ts)
    inb = n * w["dim"] * w["bits"] // 8
    val = inb / step / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": round(val, 4), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(step * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32" if w["bits"] == 32 else "f64", "data": "synthetic",
        "config": bench_config(w, n, world, seg, sbytes),
        "cpu_baseline": {"value": round(val, 4), "unit": "GB/s", "cores": cores, "kind": "port",
                         "sample": f"the full snapshot ({n} points) per step, compress + decompress, "
                                   "OpenMP C++ restatement of the reference algorithm (the reference has no "
                                   "CPU implementation)"},
        "e2e": {"value": round(val, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_e2e(args, world, w, p, host_axes, n, dev, inb, ref_out):
    """Compress + decompress through the C ABI from and to pinned host buffers,
    every copy timed.  Consecutive steps overlap their copies
    (gpz_b200.pipeline.SnapshotPipeline): each step uploads the snapshot,
    downloads its stream, uploads the stream again and downloads the
    reconstruction.  The last step's host reconstruction must equal the
    device-resident one."""
    import torch
    from gpz_b200.pipeline import SnapshotPipeline
    pipe = SnapshotPipeline(p, n, w["dim"], w["bits"], dev)
    e2e_steps = max(2, min(args.steps, 10))
    pipe.round_trips(host_axes, 2)  # warm-up
    barrier(world)
    te0 = time.perf_counter()
    nb, rx = pipe.round_trips(host_axes, e2e_steps)
    te1 = time.perf_counter()
    for h, d in zip(rx, ref_out):
        if not torch.equal(h, d.cpu()):
            raise RuntimeError("end-to-end reconstruction differs from the device-resident one")
    e2e_ms = max_over_ranks((te1 - te0) * 1e3 / e2e_steps, world)
    return world * inb / (e2e_ms * 1e-3) / 1e9, nb, e2e_steps


def strict_bound_run(gz, x, y, z, n, eb, rel):
    """The same snapshot in strict-bound mode (GPZ_FLAG_STRICT_BOUND), at the
    bench's rel 1e-4 and at abs 1e-3 with segment size 32: every point checked
    against the stated bound (gpz_verify)."""
    import numpy as np
    import torch
    cap = gz.stream_bound(n, 3, 32)
    out = torch.empty(cap, dtype=torch.uint8, device=x.device)
    scr = torch.empty(gz.compress_scratch_bytes(n), dtype=torch.uint8, device=x.device)
    sd = torch.empty(256, dtype=torch.uint8, device=x.device)
    rx, ry, rz = (torch.empty_like(x) for _ in range(3))
    res = {}
    for name, eb_s, seg, rel_mode in (("rel_1e-4", float(eb), 0, True), ("abs_1e-3_seg32", float(np.float32(1e-3)), 32, False)):
        p = gz.make_params(n, 3, 32, eb_s, seg, rel_mode, rel if rel_mode else 0.0, strict=True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        gz.compress_into(p, x, y, z, out, scr)
        e0.record()
        r = gz.compress_into(p, x, y, z, out, scr)
        e1.record()
        torch.cuda.synchronize()
        rd = gz.decompress_into(out, r.stream_bytes, 32, 3, rx, ry, rz, sd)
        hdr = gz.parse_header(out[:32].cpu().numpy().tobytes())
        v = gz.verify(x, y, z, rx, ry, rz, hdr["eb"], r.seg_size, bound=eb_s)
        res[name] = {"status": int(r.status) | int(rd.status), "eb_stated": eb_s, "eb_encoded": hdr["eb"],
                     "segment_size": int(r.seg_size), "stream_bytes": int(r.stream_bytes),
                     "over_bound": int(v.over_bound), "over_1.01eb": int(v.over_bound_tol),
                     "max_abs_err": [round(t, 9) for t in v.max_abs_err], "compress_ms": round(e0.elapsed_time(e1), 4)}
    del out, scr, rx, ry, rz
    return res


def run_ours(args):
    import numpy as np
    import torch
    import gpz_b200 as gz

    world, rank, local = dist_setup(args.gpus)
    dev = torch.device("cuda", local if world > 1 else 0)
    w = WORKLOADS[args.config]
    headline = args.config == "clustered"
    n, dim, bits = args.points or w["n"], w["dim"], w["bits"]
    dt = torch.float32 if bits == 32 else torch.float64
    x, y, z = gen_workload(w, n, (1234 if w["gen"] == "clustered" else 2024) + rank, dev)
    inb = n * dim * bits // 8
    rel_mode = w["mode"] == "rel"
    rel = typed(bits, w["e"])
    if rel_mode:
        eb, _ = gz.rel_to_abs(x, y, z, w["e"])  # the CLI's rel->abs, on the device; untimed as in the reference
    else:
        eb = rel
    p = gz.make_params(n, dim, bits, eb, w["seg"], rel_mode, rel if rel_mode else 0.0)
    cap = gz.stream_bound(n, dim, bits)
    out = torch.empty(cap, dtype=torch.uint8, device=dev)
    scr_c = torch.empty(gz.compress_scratch_bytes(n), dtype=torch.uint8, device=dev)
    scr_d = torch.empty(256, dtype=torch.uint8, device=dev)
    ox, oy = (torch.empty(n, dtype=dt, device=dev) for _ in range(2))
    oz = torch.empty(n, dtype=dt, device=dev) if dim == 3 else None
    zc, ozc = (z, oz) if dim == 3 else (x, ox)  # the ABI ignores the third axis in 2D
    stream = torch.cuda.current_stream(dev)

    # correctness gate before timing: the round trip, every point paired with
    # its own reconstruction (gpz_verify)
    r = gz.compress_into(p, x, y, zc, out, scr_c)
    rr = gz.decompress_into(out, r.stream_bytes, bits, dim, ox, oy, ozc, scr_d)
    assert r.status == 0 and rr.status == 0
    sbytes = int(r.stream_bytes)
    hdr = gz.parse_header(out[:32].cpu().numpy().tobytes())
    ver = gz.verify(x, y, z, ox, oy, oz, hdr["eb"], hdr["seg"])
    if headline:  # the headline holds the reference verifier's 1.01*eb tolerance; other workloads report
        assert ver.over_bound_tol == 0, ver.over_bound_tol
    ref_stream = out[:sbytes].clone()
    ref_rec = [t.clone() for t in (ox, oy, oz) if t is not None]
    strict = strict_bound_run(gz, x, y, z, n, eb, rel) if headline and not args.no_strict else None

    def step(evs=None):
        if evs is not None:
            evs[0].record(stream)
        gz.compress_into(p, x, y, zc, out, scr_c, sync=False)
        if evs is not None:
            evs[1].record(stream)
        gz.decompress_into(out, cap, bits, dim, ox, oy, ozc, scr_d, sync=False)
        if evs is not None:
            evs[2].record(stream)

    for _ in range(max(args.warmup, 3)):
        step()
    barrier(world)
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clk:
        barrier(world)
        t0.record(stream)
        for k in range(args.steps):
            step(evs[k])
        t1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    # the timed launches did the work: both calls of the last step report
    # success, and its stream and reconstruction equal the verified ones
    rc_, rd_ = gz.result_get(scr_c, stream), gz.result_get(scr_d, stream)
    if rc_.status != 0 or rd_.status != 0 or int(rc_.stream_bytes) != sbytes:
        raise RuntimeError(f"timed launches failed: compress {rc_.status}, decompress {rd_.status}")
    rec_now = [t for t in (ox, oy, oz) if t is not None]
    if not torch.equal(out[:sbytes], ref_stream) or not all(torch.equal(a, b) for a, b in zip(rec_now, ref_rec)):
        raise RuntimeError("timed launches produced a different stream or reconstruction")
    del ref_rec
    total_ms = max_over_ranks(t0.elapsed_time(t1), world)
    c_ms = [e[0].elapsed_time(e[1]) for e in evs]
    d_ms = [e[1].elapsed_time(e[2]) for e in evs]
    ms_step = total_ms / args.steps
    value = world * inb / (ms_step * 1e-3) / 1e9
    comp_gbs = inb / (statistics.mean(c_ms) * 1e-3) / 1e9
    dec_gbs = inb / (statistics.mean(d_ms) * 1e-3) / 1e9
    clocks = clk.summary()

    # roofline of the two codec kernels: algorithmic bytes per launch (input
    # + stream) over their mean CUDA-event durations in the timed region
    peak, peak_kind = peaks()
    alg = inb + sbytes
    achieved_c = alg / (statistics.mean(c_ms) * 1e-3) / 1e9
    achieved_d = alg / (statistics.mean(d_ms) * 1e-3) / 1e9
    tname = "float" if bits == 32 else "double"
    traffic_c = traffic_from_profile(n, "compress") if headline else None
    traffic_d = traffic_from_profile(n, "decompress") if headline else None

    # ---- end to end through the C ABI with pinned host buffers ----
    host = [t.cpu().pin_memory() for t in (x, y, z) if t is not None]
    if args.no_e2e:
        e2e_val, nb, e2e_steps = None, sbytes, 0
    else:
        e2e_val, nb, e2e_steps = run_e2e(args, world, w, p, host, n, dev, inb, rec_now)

    ref_gpu = None
    if world == 1 and rank == 0 and not args.no_reference_gpu:
        ours_stream = out[:sbytes].cpu().numpy()
        ours_rec = np.concatenate([t.cpu().numpy() for t in rec_now]).view(np.uint8)
        ref_gpu = reference_gpu_run(w, host[0], host[1], host[2] if dim == 3 else None, n, float(eb), rel,
                                    ours_stream, ours_rec, max(3, min(args.steps, 10)))
        del ours_stream, ours_rec

    cpu = None
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        ts, cores, _, _ = cpu_baseline_run(w, host[0].numpy(), host[1].numpy(),
                                           host[2].numpy() if dim == 3 else None, 1)
        cpu = {"value": round(inb / ts[0] / 1e9, 4), "unit": "GB/s", "cores": cores, "kind": "port",
               "sample": f"one compress + decompress of the same {n}-point snapshot on {cores} host threads "
                         "(OpenMP C++ restatement of the reference algorithm)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": round(ms_step, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if bits == 32 else "f64",
            "data": "synthetic (seeded generator standing in for the snapshots named in the workload)",
            "config": bench_config(w, n, world, r.seg_size, sbytes),
            "verified": {"points": int(ver.points), "over_bound": int(ver.over_bound),
                         "over_1.01eb": int(ver.over_bound_tol), "id_overflow": int(r.id_overflow),
                         "note": "default mode reproduces the reference's bytes and reconstruction, whose float "
                                 "rounding puts points just past eb (its verifier allows 1.01*eb); strict_bound "
                                 "holds eb for every point",
                         "max_abs_err": [round(v, 9) for v in ver.max_abs_err[:dim]], "eb": hdr["eb"],
                         "psnr_db": round(ver.psnr_combined, 3)},
            "compress_gbs": round(comp_gbs, 3), "decompress_gbs": round(dec_gbs, 3),
            "compress_ms": round(statistics.mean(c_ms), 4), "decompress_ms": round(statistics.mean(d_ms), 4),
            "compress_ms_min_median_max": [round(min(c_ms), 4), round(statistics.median(c_ms), 4), round(max(c_ms), 4)],
            "decompress_ms_min_median_max": [round(min(d_ms), 4), round(statistics.median(d_ms), 4),
                                             round(max(d_ms), 4)],
            "roofline": {"bound": "hbm", "kernel": f"compress_kernel<{tname},{dim}>", "achieved": round(achieved_c, 2),
                         "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved_c / peak, 4),
                         "traffic": traffic_c, "alg_bytes_per_launch": alg},
            "roofline_decompress": {"bound": "hbm",
                                    "kernel": f"decompress_kernel<{tname},{dim}>" + ("" if bits == 32 else
                                              " (fast pass + general pass)"),
                                    "achieved": round(achieved_d, 2), "peak": peak, "peak_kind": peak_kind,
                                    "unit": "GB/s", "frac": round(achieved_d / peak, 4), "traffic": traffic_d,
                                    "alg_bytes_per_launch": alg},
            # seg_sample, compress and decompress per step (float64: the
            # decompress fast pass and the general pass that follows it)
            "gpu_launches": (3 if bits == 32 else 4) * args.steps,
            "clocks": clocks,
            "e2e": None if e2e_val is None else
                   {"value": round(e2e_val, 4), "unit": "GB/s", "h2d_bytes_per_step": inb + nb,
                    "d2h_bytes_per_step": nb + inb, "steps": e2e_steps},
            "cpu_baseline": cpu,
            "reference_gpu": ref_gpu,
            "strict_bound": strict,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


BATCH_WORKLOAD = ("256 independent snapshots, sizes log-uniform in [1e4, 2e7] points, 75% 3D / 25% 2D, "
                  "85% float32 / 15% float64, each uniform i.i.d. in [0, L)^dim with L = 100 * (n / 1e6)^(1/dim) "
                  "(the 1M-point [0,100)^3 generator at the same density), rel error bound drawn from "
                  "{1e-3, 1e-4, 1e-5}, automatic segment size")


def batch_specs(count, seed):
    import math
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(round(math.exp(rng.uniform(math.log(1e4), math.log(2e7)))))
        dim = 3 if rng.random() < 0.75 else 2
        bits = 32 if rng.random() < 0.85 else 64
        rel = (1e-3, 1e-4, 1e-5)[int(rng.integers(3))]
        out.append((n, dim, bits, rel))
    return out


def run_batched(args):
    """Batched form: all snapshots compressed by one graph launch (device
    rel->abs, sampling, per-class persistent kernels) and decoded by one,
    against the same snapshots through per-snapshot calls.  Prints one JSON
    line; the stream bytes and reconstructions of both forms are compared."""
    import numpy as np
    import torch
    import gpz_b200 as gz
    from gpz_b200.batch import Batch, DecompressBatch, Snapshot, autotune
    dev = torch.device("cuda", 0)
    specs = batch_specs(args.batch, 4321)
    snaps = []
    g = torch.Generator(device=dev)
    for i, (n, dim, bits, rel) in enumerate(specs):
        g.manual_seed(1000 + i)
        L = 100.0 * (n / 1e6) ** (1.0 / dim)
        dt = torch.float32 if bits == 32 else torch.float64
        xyz = [torch.rand(n, generator=g, device=dev, dtype=dt) * L for _ in range(dim)]
        snaps.append((xyz[0], xyz[1], xyz[2] if dim == 3 else None, rel))
    inb = sum(n * dim * bits // 8 for n, dim, bits, _ in specs)
    stream = torch.cuda.current_stream(dev)

    def ev_time(fn, reps):
        for _ in range(max(args.warmup, 3)):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    # ---- batched
    b = Batch([Snapshot(x, y, z, rel_eb=rel) for x, y, z, rel in snaps])
    t_bc = ev_time(lambda: b.launch(stream), args.steps)
    res = b.results()
    assert all(r.status == 0 for r, _ in res), [r.status for r, _ in res]
    streams = b.streams()
    d = DecompressBatch(streams)
    t_bd = ev_time(lambda: d.launch(stream), args.steps)
    assert all(st == 0 for st in d.results())
    cbytes = sum(int(r.stream_bytes) for r, _ in res)

    # ---- per-snapshot calls: rel->abs on the device (a synchronising call
    # that returns the bound to the host) then compress, as a user of the
    # single-stream API does; and compress alone with the bounds known
    ebs = [eb for _, eb in res]
    plain_out = [torch.empty(gz.stream_bound(x.numel(), 3 if z is not None else 2, 32 if x.dtype == torch.float32 else 64),
                             dtype=torch.uint8, device=dev) for x, y, z, _ in snaps]
    plain_scr = [torch.empty(gz.compress_scratch_bytes(x.numel()), dtype=torch.uint8, device=dev) for x, _, _, _ in snaps]
    params = []
    for (x, y, z, rel), eb in zip(snaps, ebs):
        bits = 32 if x.dtype == torch.float32 else 64
        params.append(gz.make_params(x.numel(), 3 if z is not None else 2, bits, eb, 0, True,
                                     float(np.float32(rel)) if bits == 32 else rel))

    def plain_with_rel():
        for (x, y, z, rel), p, o, sc in zip(snaps, params, plain_out, plain_scr):
            gz.rel_to_abs(x, y, z, rel, stream)
            gz.compress_into(p, x, y, z if z is not None else x, o, sc, stream, sync=False)

    def plain_compress():
        for (x, y, z, _), p, o, sc in zip(snaps, params, plain_out, plain_scr):
            gz.compress_into(p, x, y, z if z is not None else x, o, sc, stream, sync=False)

    # the batch with the bounds given (no device rel->abs), the counterpart of
    # the compress-only per-snapshot arm
    b2 = Batch([Snapshot(x, y, z, eb=eb, rel_eb=rel, rel_mode=True) for (x, y, z, rel), eb in zip(snaps, ebs)])
    t_bc2 = ev_time(lambda: b2.launch(stream), args.steps)
    res2 = b2.results()
    same = all(r.status == 0 for r, _ in res2) and all(
        torch.equal(o, s_b) for o, s_b in zip(b2.streams(), streams))
    b2.close()
    t_pcr = ev_time(plain_with_rel, max(1, args.steps // 2))
    t_pc = ev_time(plain_compress, args.steps)
    for (x, _, _, _), o, sc, s_b in zip(snaps, plain_out, plain_scr, streams):
        r = gz.result_get(sc, stream)
        same &= r.status == 0 and r.stream_bytes == s_b.numel() and torch.equal(o[: r.stream_bytes], s_b)
    dec_out = [tuple(torch.empty_like(x) if t is not None else None for t in (x, y, z)) for x, y, z, _ in snaps]
    dscr = [torch.empty(256, dtype=torch.uint8, device=dev) for _ in snaps]

    def plain_decompress():
        for s_b, (ox, oy, oz), (x, _, z, _), sc in zip(streams, dec_out, snaps, dscr):
            dim = 3 if z is not None else 2
            gz.decompress_into(s_b, s_b.numel(), 32 if x.dtype == torch.float32 else 64, dim, ox, oy,
                               oz if dim == 3 else ox, sc, stream, sync=False)

    t_pd = ev_time(plain_decompress, args.steps)
    torch.cuda.synchronize()

    # ---- where the ceiling is: per-snapshot plain times (each call between
    # its own events, calls back to back) split at one wave of the persistent
    # compress grid.  A snapshot of a wave or more keeps every SM busy on its
    # own, so batching can at best run the smaller ones at the rate the large
    # ones reach: ceiling = plain / (plain of the large + small bytes / that
    # rate).
    def per_call_ms(calls):
        for fn in calls:
            fn()
        torch.cuda.synchronize()
        evs_ = [torch.cuda.Event(enable_timing=True) for _ in range(len(calls) + 1)]
        evs_[0].record(stream)
        for fn, e in zip(calls, evs_[1:]):
            fn()
            e.record(stream)
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in zip(evs_[:-1], evs_[1:])]

    nb_snap = [x.numel() * (3 if z is not None else 2) * (4 if x.dtype == torch.float32 else 8)
               for x, _, z, _ in snaps]
    wave_chunks = 2 * 148 * 8  # resident CTAs x SMs x chunks per CTA on a B200
    large = [x.numel() >= wave_chunks * 1024 for x, _, _, _ in snaps]
    c_calls = [(lambda x=x, y=y, z=z, p=p, o=o, sc=sc: gz.compress_into(p, x, y, z if z is not None else x, o, sc,
                                                                         stream, sync=False))
               for (x, y, z, _), p, o, sc in zip(snaps, params, plain_out, plain_scr)]
    d_calls = [(lambda s_b=s_b, ox=ox, oy=oy, oz=oz, x=x, z=z, sc=sc: gz.decompress_into(
                    s_b, s_b.numel(), 32 if x.dtype == torch.float32 else 64, 3 if z is not None else 2, ox, oy,
                    oz if z is not None else ox, sc, stream, sync=False))
               for s_b, (ox, oy, oz), (x, _, z, _), sc in zip(streams, dec_out, snaps, dscr)]

    def ceiling(ms):
        lb = sum(b for b, l in zip(nb_snap, large) if l)
        lm = sum(t for t, l in zip(ms, large) if l)
        sb = sum(b for b, l in zip(nb_snap, large) if not l)
        sm = sum(t for t, l in zip(ms, large) if not l)
        rate = lb / lm if lm > 0 else float("nan")  # bytes per ms
        best = lm + sb / rate
        return {"large_snapshots": sum(large), "large_bytes": lb, "large_plain_ms": round(lm, 3),
                "small_snapshots": len(large) - sum(large), "small_bytes": sb, "small_plain_ms": round(sm, 3),
                "large_rate_gbs": round(rate / 1e6, 2), "best_case_ms": round(best, 3),
                "ceiling_speedup": round((lm + sm) / best, 3)}

    ceil_c = ceiling(per_call_ms(c_calls))
    ceil_d = ceiling(per_call_ms(d_calls))
    for (ox, oy, oz), (bx, by, bz) in zip(dec_out, d.outputs):
        for a, c in ((ox, bx), (oy, by), (oz, bz)):
            if a is not None:
                same &= torch.equal(a.view(torch.uint8), c.view(torch.uint8))
    # ---- autotuned segment sizes: the batch and the per-snapshot calls with
    # the same (fixed) segment sizes
    tsnaps = [Snapshot(x, y, z, rel_eb=rel) for x, y, z, rel in snaps]
    tt0 = time.perf_counter()
    recs = autotune(tsnaps, stream=stream)
    tune_s = time.perf_counter() - tt0
    bt = Batch(tsnaps)
    t_bt = ev_time(lambda: bt.launch(stream), args.steps)
    rt = bt.results()
    tuned_streams = bt.streams()
    tuned_bytes = sum(int(r.stream_bytes) for r, _ in rt)
    tparams = []
    for (x, y, z, rel), snap, eb in zip(snaps, tsnaps, ebs):
        bits = 32 if x.dtype == torch.float32 else 64
        p = gz.make_params(x.numel(), 3 if z is not None else 2, bits, eb, snap.seg_size, True,
                           float(np.float32(rel)) if bits == 32 else rel)
        p.flags |= gz.GPZ_FLAG_SEG_FIXED
        tparams.append(p)

    def plain_tuned():
        for (x, y, z, rel), p, o, sc in zip(snaps, tparams, plain_out, plain_scr):
            gz.rel_to_abs(x, y, z, rel, stream)
            gz.compress_into(p, x, y, z if z is not None else x, o, sc, stream, sync=False)

    t_ptr = ev_time(plain_tuned, max(1, args.steps // 2))
    for o, sc, s_b in zip(plain_out, plain_scr, tuned_streams):
        r = gz.result_get(sc, stream)
        same &= r.status == 0 and r.stream_bytes == s_b.numel() and torch.equal(o[: r.stream_bytes], s_b)
    segs_default = [int(r.seg_size) for r, _ in res]
    segs_tuned = [s.seg_size for s in tsnaps]
    bt.close()
    gbs = lambda ms: round(inb / (ms * 1e-3) / 1e9, 2)
    line = {
        "metric": "batched compress / decompress aggregate GB/s (input bytes) vs per-snapshot calls, 1 B200",
        "unit": "GB/s", "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3), "higher_is_better": True,
        "data": "synthetic", "config": {"workload": BATCH_WORKLOAD, "snapshots": len(specs), "points": sum(s[0] for s in specs),
                                        "input_bytes": inb, "stream_bytes": cbytes},
        "batched": {"rel_and_compress_ms": round(t_bc, 3), "rel_and_compress_gbs": gbs(t_bc),
                    "compress_ms": round(t_bc2, 3), "compress_gbs": gbs(t_bc2), "decompress_ms": round(t_bd, 3),
                    "decompress_gbs": gbs(t_bd), "device_bytes": b.device_bytes},
        "plain": {"rel_and_compress_ms": round(t_pcr, 3), "rel_and_compress_gbs": gbs(t_pcr),
                  "compress_ms": round(t_pc, 3), "compress_gbs": gbs(t_pc),
                  "decompress_ms": round(t_pd, 3), "decompress_gbs": gbs(t_pd)},
        "speedup": {"rel_and_compress": round(t_pcr / t_bc, 3), "compress": round(t_pc / t_bc2, 3),
                    "decompress": round(t_pd / t_bd, 3)},
        "autotuned": {"rel_and_compress_ms": round(t_bt, 3), "rel_and_compress_gbs": gbs(t_bt),
                      "plain_rel_and_compress_ms": round(t_ptr, 3), "speedup": round(t_ptr / t_bt, 3),
                      "stream_bytes": tuned_bytes, "stream_bytes_default_seg": cbytes,
                      "ratio_gain": round(cbytes / tuned_bytes, 4), "tune_seconds": round(tune_s, 3),
                      "segments_changed": sum(a != b for a, b in zip(segs_default, segs_tuned)),
                      "candidates": [1, 2, 4, 8, 16, 32, 64, 128], "sample_points": 1 << 17},
        "identical_output": bool(same),
        "ceiling": {"note": "snapshots of at least one wave of the persistent compress grid (2 CTAs x 148 SMs x 8 "
                            "chunks = 2,424,832 points) keep the GPU busy alone; the best a batch can do is run "
                            "the smaller ones at the large ones' rate",
                    "wave_points": wave_chunks * 1024, "compress": ceil_c, "decompress": ceil_d},
    }
    b.close()
    d.close()
    print(json.dumps(line), flush=True)


SERVE_WORKLOAD = ("Poisson arrivals at the given rates, 70% compress / 30% decompress of previously produced "
                  "streams, sizes log-uniform in [1e5, 5e7] points, 3D, 80% float32 / 20% float64, rel error "
                  "bound drawn from {1e-3, 1e-4}; requests draw from a pool of 48 resident snapshots")


def run_served(args):
    """Served form: a request server (continuous batching, 120 GB budget)
    against the plain per-request path (one synchronous call per request, in
    arrival order) on the same Poisson arrival schedule.  Latency = arrival to
    completion; GB/s = input bytes / (first arrival to last completion)."""
    import math
    import threading
    import numpy as np
    import torch
    import gpz_b200 as gz
    from gpz_b200.serve import Server
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(777)
    pool = []
    g = torch.Generator(device=dev)
    for i in range(48):
        n = int(round(math.exp(rng.uniform(math.log(1e5), math.log(5e7)))))
        bits = 32 if rng.random() < 0.8 else 64
        rel = (1e-3, 1e-4)[int(rng.integers(2))]
        g.manual_seed(5000 + i)
        L = 100.0 * (n / 1e6) ** (1.0 / 3)
        dt = torch.float32 if bits == 32 else torch.float64
        x, y, z = (torch.rand(n, generator=g, device=dev, dtype=dt) * L for _ in range(3))
        eb, _ = gz.rel_to_abs(x, y, z, rel)
        st, r = gz.compress(x, y, z, eb=eb, rel_mode=True, rel_eb=rel)
        pool.append(dict(x=x, y=y, z=z, n=n, bits=bits, rel=rel, stream=st.clone(),
                         header=gz.parse_header(st[:32].cpu().numpy().tobytes()), inb=3 * n * bits // 8))
    torch.cuda.synchronize()
    scr = torch.empty(gz.compress_scratch_bytes(max(p["n"] for p in pool)), dtype=torch.uint8, device=dev)
    outc = torch.empty(max(gz.stream_bound(p["n"], 3, p["bits"]) for p in pool), dtype=torch.uint8, device=dev)
    outd = [torch.empty(max(p["n"] for p in pool), dtype=torch.float64, device=dev) for _ in range(3)]
    dscr = torch.empty(256, dtype=torch.uint8, device=dev)

    def plain_one(req):
        p = pool[req[1]]
        if req[0] == "c":
            eb, _ = gz.rel_to_abs(p["x"], p["y"], p["z"], p["rel"])
            prm = gz.make_params(p["n"], 3, p["bits"], eb, 0, True, p["rel"])
            r = gz.compress_into(prm, p["x"], p["y"], p["z"], outc, scr)
            assert r.status == 0
        else:
            dt = torch.float32 if p["bits"] == 32 else torch.float64
            o = [t.view(torch.uint8)[: p["n"] * p["bits"] // 8].view(dt) for t in outd]
            r = gz.decompress_into(p["stream"], p["stream"].numel(), p["bits"], 3, o[0], o[1], o[2], dscr)
            assert r.status == 0

    results = {}
    for rate in args.rates:
        count = args.requests
        arr = np.cumsum(rng.exponential(1.0 / rate, count))
        reqs = [("c" if rng.random() < 0.7 else "d", int(rng.integers(len(pool)))) for _ in range(count)]
        inb = sum(pool[k]["inb"] for _, k in reqs)
        # ---- served
        srv = Server(hbm_budget=120 << 30, streams=args.serve_streams, max_batch=64, overlap=args.overlap)
        lat, tickets = [0.0] * count, [None] * count
        done_at = [0.0] * count
        t0 = time.perf_counter()

        def consumer():
            for i in range(count):
                while tickets[i] is None:
                    time.sleep(0.0001)
                c = srv.wait(tickets[i], timeout_ms=600_000)
                assert c.status == 0, c.status
                done_at[i] = time.perf_counter()
                lat[i] = c.total_ms
                srv.release(tickets[i])

        th = threading.Thread(target=consumer)
        th.start()
        for i, (op, k) in enumerate(reqs):
            now = time.perf_counter() - t0
            if arr[i] > now:
                time.sleep(arr[i] - now)
            p = pool[k]
            if op == "c":
                tickets[i] = srv.submit_compress(p["x"], p["y"], p["z"], rel_eb=p["rel"])
            else:
                tickets[i] = srv.submit_decompress(p["stream"], p["header"])
        th.join()
        span = max(done_at) - t0 - arr[0]
        st = srv.stats()
        srv.close()
        # ---- plain: one synchronous call per request, in arrival order
        platency = []
        t0 = time.perf_counter()
        for i, req in enumerate(reqs):
            now = time.perf_counter() - t0
            if arr[i] > now:
                time.sleep(arr[i] - now)
            plain_one(req)
            platency.append((time.perf_counter() - t0 - arr[i]) * 1e3)
        pspan = time.perf_counter() - t0 - arr[0]
        results[str(rate)] = {
            "requests": count, "input_bytes": inb,
            "served": {"p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3),
                       "gbs": round(inb / span / 1e9, 2), "batches": int(st.batches),
                       "mean_batch": round(count / max(1, st.batches), 2)},
            "plain": {"p50_ms": round(float(np.percentile(platency, 50)), 3),
                      "p99_ms": round(float(np.percentile(platency, 99)), 3), "gbs": round(inb / pspan / 1e9, 2)},
        }
    line = {"metric": "served p50/p99 latency (ms) and aggregate GB/s vs per-request calls, 1 B200", "unit": "ms",
            "n_gpus": 1, "higher_is_better": False, "data": "synthetic",
            "config": {"workload": SERVE_WORKLOAD, "hbm_budget_bytes": 120 << 30, "streams": args.serve_streams,
                       "overlap": bool(args.overlap), "max_batch": 64,
                       "pool_points": sum(p["n"] for p in pool)},
            "rates": results}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end timing")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip timing the reference's own GPU build on the same snapshot")
    ap.add_argument("--no-strict", action="store_true", help="skip the strict-bound runs")
    ap.add_argument("--batched", action="store_true",
                    help="time the batched form (many snapshots per graph launch) against per-snapshot calls")
    ap.add_argument("--batch", type=int, default=256, help="snapshots in the batched workload")
    ap.add_argument("--served", action="store_true",
                    help="time the request server against per-request calls on a Poisson arrival schedule")
    ap.add_argument("--rates", type=float, nargs="+", default=[50.0, 200.0, 800.0])
    ap.add_argument("--requests", type=int, default=300, help="requests per arrival rate")
    ap.add_argument("--serve-streams", type=int, default=2)
    ap.add_argument("--overlap", action="store_true", help="let served batches run concurrently")
    ap.add_argument("--points", type=int, default=0,
                    help="points per GPU (smaller cases for profiler captures; 0: the workload's size)")
    ap.add_argument("--config", choices=sorted(WORKLOADS), default="clustered",
                    help="workload (default: the 143.7M-point clustered float32 snapshot at rel 1e-4)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.batched:
        run_batched(args)
    elif args.served:
        run_served(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
