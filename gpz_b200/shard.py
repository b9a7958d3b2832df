"""Sharded compression of one snapshot across the ranks of a torch.distributed
group (one GPU per rank).

The reference compresses on one GPU.  Its 1024-point chunks are encoded
independently given the error bound and the segment size, so an array cut into
chunk-aligned shards can be encoded shard by shard -- each shard as an ordinary
stream with the bound and segment size agreed for the whole array -- and the
pieces stitched into exactly the bytes a single-GPU run produces:

    header | offset table (G x u64) | meta (G records) | payloads

Shard r owns chunks [c_r, c_{r+1}): its offset-table entries (rebased by the
payload bytes of shards before it), its meta records and its payload go to
known byte ranges of the whole stream.  The only collectives are tiny:

* relative bound: all-reduce of the six per-axis minima / maxima
  (findMinimumValues + convertRelEb, reference include/utils.cuh:44-65,
  src/main.cpp:35-55), then the conversion on the host;
* automatic segment size: all-reduce (max) of the six accumulators of
  computeSegSize's sample windows (src/cudaWarpCompress.cu:1424-1557), then
  its rules on the host -- the same code the single-GPU sampling kernel runs;
* an all-gather of the shards' payload sizes.

After that the shards' pieces are independent.  `gather_stream` moves them
into the root's whole-stream buffer with point-to-point sends (NCCL over
NVLink on GPUs); `stitch` does the same assembly from host bytes.

The local work of a rank goes through a codec object: `GpuCodec` runs the
library's kernels (gpz_rel_to_abs, gpz_sample_minmax, gpz_compress with the
segment size fixed).  The stitching logic takes the codec as a parameter, so the
same code is exercised by multi-process CPU tests with a host codec.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

CHUNK = 1024
HDR = {32: 24, 64: 32}
META = {32: 36, 64: 64}


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Chunk-aligned [begin, begin + count) of an n-point array owned by `rank`
    (chunks split as evenly as possible; every shard but the last holds whole
    chunks)."""
    g = (n + CHUNK - 1) // CHUNK
    c0, c1 = (g * rank) // world, (g * (rank + 1)) // world
    b, e = c0 * CHUNK, min(c1 * CHUNK, n)
    return b, max(0, e - b)


@dataclass
class ShardLayout:
    """Where this rank's pieces go in the whole stream (byte offsets)."""
    n_total: int
    bits: int
    chunk0: int         # first chunk of the shard
    chunks: int         # chunks in the shard
    payload_base: int   # payload bytes of the shards before this one
    payload: int        # this shard's payload bytes
    total_bytes: int    # size of the whole stream
    sizes: tuple = ()   # payload bytes of every shard, in rank order

    @property
    def g_total(self) -> int:
        return (self.n_total + CHUNK - 1) // CHUNK

    @property
    def table_range(self) -> tuple[int, int]:
        a = HDR[self.bits] + 8 * self.chunk0
        return a, a + 8 * self.chunks

    @property
    def meta_range(self) -> tuple[int, int]:
        a = HDR[self.bits] + 8 * self.g_total + META[self.bits] * self.chunk0
        return a, a + META[self.bits] * self.chunks

    @property
    def payload_range(self) -> tuple[int, int]:
        a = HDR[self.bits] + (8 + META[self.bits]) * self.g_total + self.payload_base
        return a, a + self.payload


def _lib():
    from . import lib
    return lib()


def rel_abs_from_minmax(bits: int, mm6, rel: float) -> float:
    """convertRelEb on combined per-axis minima / maxima (library host code)."""
    mm = (ctypes.c_double * 6)(*[float(v) for v in mm6])
    eb = ctypes.c_double(0.0)
    rc = _lib().gpz_rel_abs_from_minmax(bits, mm, float(rel), ctypes.byref(eb))
    if rc:
        raise RuntimeError(f"gpz_rel_abs_from_minmax failed ({rc})")
    return eb.value


def decide_seg(bits: int, dim: int, acc6, seg_in: int, rel_mode: bool, rel_eb: float, eb: float,
               flags: int = 0) -> tuple[int, int]:
    """computeSegSize's rules on combined sample accumulators (library host code)."""
    acc = (ctypes.c_uint64 * 6)(*[int(v) for v in acc6])
    seg, adj = ctypes.c_uint32(0), ctypes.c_uint32(0)
    rc = _lib().gpz_decide_seg(bits, dim, acc, seg_in, 1 if rel_mode else 0, float(rel_eb), float(eb), flags,
                               ctypes.byref(seg), ctypes.byref(adj))
    if rc:
        raise RuntimeError(f"gpz_decide_seg failed ({rc})")
    return seg.value, adj.value


def _all_reduce(values, op, group):
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    # float64 / int64 explicitly: torch's default float tensor is float32
    dt = torch.int64 if all(isinstance(v, int) for v in values) else torch.float64
    t = torch.tensor(values, dtype=dt, device=dev)
    dist.all_reduce(t, op=op, group=group)
    return t.cpu().tolist()


def agree_bound(codec, rel: float, group) -> float:
    """Absolute bound of the whole array from a relative one."""
    import torch.distributed as dist
    mm = codec.minmax()
    lo = _all_reduce([float(v) for v in mm[:3]], dist.ReduceOp.MIN, group)
    hi = _all_reduce([float(v) for v in mm[3:]], dist.ReduceOp.MAX, group)
    return rel_abs_from_minmax(codec.bits, lo + hi, rel)


def agree_seg(codec, seg_in: int, rel_mode: bool, rel_eb: float, eb: float, group, flags: int = 0):
    """Segment size of the whole array: the shards' sample accumulators are
    combined with an unsigned max (as int64 with the top bit flipped, which keeps
    the order) and the rules applied once."""
    import torch.distributed as dist
    def to_signed(u: int) -> int:  # unsigned order -> int64 order
        s = int(u) ^ (1 << 63)
        return s - (1 << 64) if s >= (1 << 63) else s

    def to_unsigned(v: int) -> int:
        return ((int(v) + (1 << 64)) % (1 << 64)) ^ (1 << 63)

    red = _all_reduce([to_signed(v) for v in codec.sample_acc()], dist.ReduceOp.MAX, group)
    combined = [to_unsigned(v) for v in red]
    return decide_seg(codec.bits, codec.dim, combined, seg_in, rel_mode, rel_eb, eb, flags)


def compress_sharded(codec, eb: float, seg: int, group) -> ShardLayout:
    """Encodes this rank's shard with the agreed bound and segment size, learns
    the other shards' payload sizes and rebases its offset-table slice.  The
    codec keeps the shard stream; the returned layout says where its pieces go."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    payload = int(codec.compress(eb, seg))
    sizes = _all_gather_int(payload, group)
    base = sum(sizes[:rank])
    codec.rebase_offsets(base)
    return layout_of(codec.n_total, codec.bits, rank, world, sizes)


def layout_of(n_total: int, bits: int, rank: int, world: int, sizes) -> ShardLayout:
    """Layout of shard `rank` given every shard's payload size."""
    b, c = shard_range(n_total, rank, world)
    g_total = (n_total + CHUNK - 1) // CHUNK
    return ShardLayout(n_total, bits, b // CHUNK, (c + CHUNK - 1) // CHUNK, sum(sizes[:rank]), sizes[rank],
                       HDR[bits] + (8 + META[bits]) * g_total + sum(sizes), tuple(sizes))


def _all_gather_int(v: int, group) -> list[int]:
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.int64, device=dev)
    out = [torch.zeros_like(t) for _ in range(dist.get_world_size(group))]
    dist.all_gather(out, t, group=group)
    return [int(o.item()) for o in out]


def stitch(pieces: list[tuple[ShardLayout, bytes]], header: bytes) -> bytes:
    """Whole stream from the shards' local streams (each a complete stream of
    its shard, offsets already rebased) -- the assembly a writer or a gather
    does; `header` is any shard's header with the total point count."""
    lay0 = pieces[0][0]
    out = bytearray(lay0.total_bytes)
    hb = HDR[lay0.bits]
    out[:hb] = header[:hb]
    for lay, s in pieces:
        g, mb = lay.chunks, META[lay.bits]
        t0, t1 = lay.table_range
        m0, m1 = lay.meta_range
        p0, p1 = lay.payload_range
        out[t0:t1] = s[hb:hb + 8 * g]
        out[m0:m1] = s[hb + 8 * g:hb + 8 * g + mb * g]
        out[p0:p1] = s[hb + (8 + mb) * g:hb + (8 + mb) * g + lay.payload]
    return bytes(out)


def gather_stream(local, lay: ShardLayout, group, root: int = 0):
    """Collects the whole stream on `root` as one uint8 tensor on the device of
    `local` (this rank's shard stream, offsets already rebased; a CUDA tensor
    under NCCL, a CPU tensor under gloo).  Every other rank sends its offset
    slice, meta records and payload straight into their byte ranges of the
    root's buffer (point-to-point sends; sizes are known from the size
    all-gather, so the root posts exactly matching receives).  Returns None on
    the other ranks."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    hb, mb = HDR[lay.bits], META[lay.bits]

    def ranges(l: ShardLayout):
        """(source range in the shard stream, target range in the whole stream)
        of the offset slice, the meta records and the payload."""
        g = l.chunks
        src = [(hb, hb + 8 * g), (hb + 8 * g, hb + (8 + mb) * g), (hb + (8 + mb) * g, hb + (8 + mb) * g + l.payload)]
        return [(s_, d_) for s_, d_ in zip(src, (l.table_range, l.meta_range, l.payload_range)) if s_[1] > s_[0]]

    def peer(r):
        return dist.get_global_rank(group, r) if group is not None else r

    if rank != root:
        for (a, b), _ in ranges(lay):
            dist.send(local[a:b].contiguous(), dst=peer(root), group=group)
        return None
    out = torch.empty(lay.total_bytes, dtype=torch.uint8, device=local.device)
    out[:hb] = local[:hb]
    out[4:12] = torch.tensor(list(int(lay.n_total).to_bytes(8, "little")), dtype=torch.uint8)
    for r in range(world):
        for (a, b), (c, d) in ranges(layout_of(lay.n_total, lay.bits, r, world, lay.sizes)):
            if r == root:
                out[c:d] = local[a:b]
            else:
                dist.recv(out[c:d], src=peer(r), group=group)
    return out


def whole_header(local_header: bytes, n_total: int) -> bytes:
    """A shard's header with the whole array's point count (u64 at byte 4)."""
    h = bytearray(local_header)
    h[4:12] = int(n_total).to_bytes(8, "little")
    return bytes(h)


class GpuCodec:
    """One rank's shard on its GPU: x, y, z are CUDA tensors holding points
    [begin, begin + count) of an n_total-point array."""

    def __init__(self, x, y, z, n_total: int, begin: int, dim: int = 3):
        import torch
        from . import compress_scratch_bytes, stream_bound
        self.x, self.y, self.z = x, y, (z if dim == 3 else y)
        self.n_total, self.begin, self.count, self.dim = n_total, begin, x.numel(), dim
        self.bits = 32 if x.dtype == torch.float32 else 64
        dev = x.device
        self.out = torch.empty(max(stream_bound(self.count, dim, self.bits), 64), dtype=torch.uint8, device=dev)
        self.scratch = torch.empty(compress_scratch_bytes(self.count), dtype=torch.uint8, device=dev)
        self.small = torch.empty(256, dtype=torch.uint8, device=dev)
        self.stream_bytes = 0

    def _stream(self):
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream(self.x.device).cuda_stream)

    def minmax(self):
        from . import rel_to_abs
        _, mm = rel_to_abs(self.x, self.y, self.z if self.dim == 3 else None, 1.0)
        return list(mm)

    def sample_acc(self):
        acc = (ctypes.c_uint64 * 6)()
        rc = _lib().gpz_sample_minmax(self.bits, self.dim, self.n_total, self.begin, self.count, self.x.data_ptr(),
                                      self.y.data_ptr(), self.z.data_ptr(), self.small.data_ptr(),
                                      self.small.numel(), acc, self._stream())
        if rc:
            raise RuntimeError(f"gpz_sample_minmax failed ({rc})")
        return list(acc)

    def compress(self, eb: float, seg: int) -> int:
        from . import Params, Result, GPZ_FLAG_SEG_FIXED
        p = Params(self.bits, self.dim, self.count, float(eb), 0.0, 0, int(seg), GPZ_FLAG_SEG_FIXED, 0)
        r = Result()
        rc = _lib().gpz_compress(ctypes.byref(p), self.x.data_ptr(), self.y.data_ptr(), self.z.data_ptr(),
                                 self.out.data_ptr(), self.out.numel(), self.scratch.data_ptr(),
                                 self.scratch.numel(), ctypes.byref(r), self._stream())
        if rc or r.status:
            raise RuntimeError(f"gpz_compress failed ({rc or r.status})")
        self.stream_bytes = r.stream_bytes
        g = (self.count + CHUNK - 1) // CHUNK
        return r.stream_bytes - HDR[self.bits] - (8 + META[self.bits]) * g

    def rebase_offsets(self, base: int) -> None:
        if base:
            g = (self.count + CHUNK - 1) // CHUNK
            hb = HDR[self.bits]
            tab = self.out[hb:hb + 8 * g].view(__import__("torch").int64)
            tab += base

    def local_tensor(self):
        """The shard stream in device memory (the argument of gather_stream)."""
        return self.out[:self.stream_bytes]

    def local_stream(self) -> bytes:
        return self.local_tensor().cpu().numpy().tobytes()
