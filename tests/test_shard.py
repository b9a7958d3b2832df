"""Sharded compression of one array (gpz_b200.shard): chunk-aligned shards
encoded with the bound and segment size agreed over the group, stitched into
exactly the single-run stream.

CPU: two gloo ranks run the collective logic (bound, segment size, payload
offsets, the point-to-point gather) with a host codec built on the oracle, and
rank 0's whole stream is compared byte for byte with the oracle's whole-array
stream.  GPU: the library
pieces (shard sampling, host segment rules, fixed-segment compress, offset
rebasing) on one GPU, shard by shard, against the library's own single-call
stream."""
import os
import socket

import numpy as np
import pytest

from gpz_b200 import shard as sh


# ------------------------------------------------------------ host codec (CPU)

def _ord(v, bits):
    u = np.asarray(v, np.float32 if bits == 32 else np.float64).view(np.uint32 if bits == 32 else np.uint64)
    top = np.uint32(0x80000000) if bits == 32 else np.uint64(1 << 63)
    return np.where(u & top, ~u, u | top)


class HostCodec:
    """The test's stand-in for GpuCodec: the same local quantities from the
    host arrays, the oracle as the shard encoder."""

    def __init__(self, x, y, z, n_total, begin, dim):
        self.x, self.y, self.z = x, y, z
        self.n_total, self.begin, self.count, self.dim = n_total, begin, len(x), dim
        self.bits = 32 if x.dtype == np.float32 else 64
        self.stream = None

    def minmax(self):
        lim = np.finfo(np.float32).max  # the host scan starts from float limits (include/utils.cuh:48-53)
        mm = []
        for a in (self.x, self.y, self.z if self.dim == 3 else np.zeros(1, self.x.dtype)):
            a = a[~np.isnan(a)]
            mm.append((min(float(a.min()), lim) if len(a) else lim, max(float(a.max()), -lim) if len(a) else -lim))
        return [m[0] for m in mm] + [m[1] for m in mm]

    def sample_acc(self):
        n, L, B = self.n_total, 256, 1024
        stride = max((n - L) // B, 1)
        acc = [0] * 6
        axes = [self.x, self.y, self.z][:self.dim]
        for w in range(B):
            st = w * stride
            for d, a in enumerate(axes):
                if st + L > n:
                    vals = np.zeros(1, a.dtype)
                else:
                    lo, hi = max(st, self.begin), min(st + L, self.begin + self.count)
                    if lo >= hi:
                        continue
                    vals = a[lo - self.begin:hi - self.begin]
                    vals = vals[~np.isnan(vals)]
                    if not len(vals):
                        continue
                o = _ord(vals, self.bits)
                mask = (1 << self.bits) - 1
                acc[2 * d] = max(acc[2 * d], int((~o).max()) & mask)
                acc[2 * d + 1] = max(acc[2 * d + 1], int(o.max()))
        return acc

    def compress(self, eb, seg):
        from oracle import pyoracle as po
        self.stream = bytearray(po.compress(self.x, self.y, self.z, self.dim, eb, seg))
        g = (self.count + 1023) // 1024
        return len(self.stream) - sh.HDR[self.bits] - (8 + sh.META[self.bits]) * g

    def local_tensor(self):
        import torch
        return torch.from_numpy(np.frombuffer(bytes(self.stream), np.uint8).copy())

    def rebase_offsets(self, base):
        g = (self.count + 1023) // 1024
        hb = sh.HDR[self.bits]
        t = np.frombuffer(self.stream, np.uint64, count=g, offset=hb).copy() + np.uint64(base)
        self.stream[hb:hb + 8 * g] = t.tobytes()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, case, q):
    import torch.distributed as dist
    from oracle import pyoracle as po
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        kind, n, dim, bits, mode, e, seg_in = case
        dt = np.float32 if bits == 32 else np.float64
        x, y, z = po.generate(kind, n, dim, 0.0, 500.0, 7, dt)
        b, c = sh.shard_range(n, rank, world)
        codec = HostCodec(x[b:b + c], y[b:b + c], z[b:b + c], n, b, dim)
        eb = sh.agree_bound(codec, e, None) if mode == "rel" else e
        seg, adj = sh.agree_seg(codec, seg_in, mode == "rel", e, eb, None)
        lay = sh.compress_sharded(codec, eb, seg, None)
        got = [None] * world
        dist.all_gather_object(got, (lay, bytes(codec.stream)))
        gathered = sh.gather_stream(codec.local_tensor(), lay, None, root=0)
        if rank == 0:
            whole = sh.stitch(got, sh.whole_header(got[0][1][:sh.HDR[bits]], n))
            assert bytes(gathered.numpy().tobytes()) == whole
            eb1 = po.rel_to_abs(x, y, z, e) if mode == "rel" else e
            seg1, adj1 = po.seg_size(x, y, z, dim, seg_in, mode == "rel", e, eb1, False)
            ref = po.compress(x, y, z, dim, eb1, seg1)
            q.put((eb == eb1, (seg, adj) == (seg1, adj1), whole == bytes(ref), len(whole), len(ref)))
    except Exception as ex:  # report instead of hanging the other rank
        q.put(repr(ex))
        raise
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case,world", [
    ((1, 50_000, 3, 32, "rel", 1e-4, 0), 2),     # clustered f32 3D, automatic segment size
    ((0, 33_333, 2, 64, "rel", 1e-5, 0), 2),     # uniform f64 2D, ragged last chunk
    ((2, 40_960, 3, 64, "abs", 0.02, 16), 2),    # lattice f64 3D, given segment size
    ((1, 5_000, 2, 32, "rel", 1e-3, 0), 3),      # 5 chunks over 3 ranks
])
def test_ranks_stitch_to_single_run_bytes(case, world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, case, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = q.get(timeout=10)
    assert not isinstance(res, str), res
    same_eb, same_seg, same_bytes, n1, n2 = res
    assert same_eb and same_seg
    assert same_bytes, (n1, n2)


def test_shard_ranges_cover_the_array():
    for n in (1, 1023, 1024, 1025, 100_000, 143_735_721):
        for world in (1, 2, 3, 8):
            spans = [sh.shard_range(n, r, world) for r in range(world)]
            pos = 0
            for b, c in spans:
                assert b == pos or c == 0
                assert b % 1024 == 0
                pos = b + c if c else pos
            assert pos == n


# --------------------------------------------------------------------- GPU

@pytest.mark.gpu
@pytest.mark.parametrize("bits,dim,rel", [(32, 3, 1e-4), (64, 2, 1e-5)])
def test_gpu_shards_stitch_to_single_call_stream(bits, dim, rel):
    """Three shards encoded one after another on the GPU with the agreed bound
    and segment size stitch to the single gpz_compress stream."""
    import torch
    import gpz_b200 as gz
    from oracle import pyoracle as po
    dt = np.float32 if bits == 32 else np.float64
    n = 123_457
    x, y, z = (torch.from_numpy(a.copy()).cuda() for a in po.generate(1, n, dim, 0.0, 800.0, 5, dt))
    zz = z if dim == 3 else None
    world = 3
    codecs = []
    for r in range(world):
        b, c = sh.shard_range(n, r, world)
        codecs.append(sh.GpuCodec(x[b:b + c], y[b:b + c], z[b:b + c], n, b, dim))
    # the collectives, done by hand
    mms = [cd.minmax() for cd in codecs]
    lo = [min(m[i] for m in mms) for i in range(3)]
    hi = [max(m[3 + i] for m in mms) for i in range(3)]
    eb = sh.rel_abs_from_minmax(bits, lo + hi, rel)
    accs = [cd.sample_acc() for cd in codecs]
    seg, adj = sh.decide_seg(bits, dim, [max(a[i] for a in accs) for i in range(6)], 0, True, rel, eb)
    sizes = [cd.compress(eb, seg) for cd in codecs]
    pieces = []
    for r, cd in enumerate(codecs):
        base = sum(sizes[:r])
        cd.rebase_offsets(base)
        lay = sh.ShardLayout(n, bits, cd.begin // 1024, (cd.count + 1023) // 1024, base, sizes[r], 0)
        lay.total_bytes = sh.HDR[bits] + (8 + sh.META[bits]) * lay.g_total + sum(sizes)
        pieces.append((lay, cd.local_stream()))
    whole = sh.stitch(pieces, sh.whole_header(pieces[0][1][:sh.HDR[bits]], n))
    eb1, _ = gz.rel_to_abs(x, y, zz, rel)
    assert eb == eb1
    stream, res = gz.compress(x, y, zz, eb=eb1, seg_size=0, rel_mode=True, rel_eb=float(dt(rel)))
    assert (seg, adj) == (res.seg_size, res.adjusted)
    assert whole == stream.cpu().numpy().tobytes()
