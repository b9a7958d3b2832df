"""Host-memory snapshots through the codec with the PCIe copies overlapped.

The CLI path of GPZ (src/main.cpp:283-360 compress, :400-450 decompress)
copies a snapshot to the device, runs the codec and copies the result back,
one step after another.  For a sequence of snapshots held in pinned host
memory, `SnapshotPipeline` keeps two device buffer sets and separate CUDA
streams for uploads, the codec and downloads, so that the upload of the next
snapshot and the download of the previous one run while the current one is
encoded or decoded.  Every step still moves its own bytes: the snapshot up,
the stream down (exactly `stream_bytes`), the stream up again and the
reconstruction down.

Stages per step i (slot k = i % 2), ordered by events.  All uploads share
one stream and all downloads another: copies on separate streams of one
direction are not interleaved by the copy engines (a ready stream copy waited
behind every queued snapshot upload), so the queue order is set here.  The
host issues step i's stream download and upload before the next snapshot's
transfers, and the reconstruction download of step i-1 after the stream
download of step i, so that each step's dependent chain (down, up,
decompress) runs ahead of the bulk copies:

    upload      host snapshot -> dX[k]            waits: compress of step i-2 done with dX[k]
    compress    dX[k] -> out[k]                    waits: upload; stream download of step i-2
    size        host reads the stream size         (the one host wait per step; posted to
                                                   pinned memory by the device, gpz_result_post)
    down        out[k][:nb] -> pinned hs[k]        waits: compress; stream upload of step i-2
    up          hs[k][:nb] -> din[k]               waits: down; decompress of step i-2
    decompress  din[k] -> oX[k]                    waits: up; reconstruction download of step i-2
    fetch       oX[k] -> pinned rX[k]              waits: decompress
"""
from __future__ import annotations

import gpz_b200 as gz


class SnapshotPipeline:
    """Round trips of float32 / float64 snapshots between pinned host memory
    and the codec with copy / compute overlap across consecutive steps.

    params: a `gz.Params` for snapshots of `n` points (`gz.make_params`)."""

    def __init__(self, params, n: int, dim: int, float_bits: int, device=None):
        torch = gz._torch()
        if dim not in (2, 3) or float_bits not in (32, 64):
            raise gz.GpzError(gz.GPZ_EINVAL, "SnapshotPipeline: dim must be 2 or 3, float_bits 32 or 64")
        self.p, self.n, self.dim, self.bits = params, n, dim, float_bits
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.dev = dev
        dt = torch.float32 if float_bits == 32 else torch.float64
        cap = gz.stream_bound(n, dim, float_bits)
        self.cap = cap
        ax = dim

        def dev_axes():
            return [torch.empty(n, dtype=dt, device=dev) for _ in range(ax)]

        def host_axes():
            return [torch.empty(n, dtype=dt).pin_memory() for _ in range(ax)]

        self.dX = [dev_axes() for _ in range(2)]
        self.out = [torch.empty(cap, dtype=torch.uint8, device=dev) for _ in range(2)]
        self.din = [torch.empty(cap, dtype=torch.uint8, device=dev) for _ in range(2)]
        self.oX = [dev_axes() for _ in range(2)]
        self.hs = [torch.empty(cap, dtype=torch.uint8).pin_memory() for _ in range(2)]
        self.rX = [host_axes() for _ in range(2)]
        self.scr_c = [torch.empty(gz.compress_scratch_bytes(n), dtype=torch.uint8, device=dev) for _ in range(2)]
        self.scr_d = [torch.empty(256, dtype=torch.uint8, device=dev) for _ in range(2)]
        # compress results land here through gpz_result_post (no copy engine)
        self.res = [torch.zeros(64, dtype=torch.uint8).pin_memory() for _ in range(2)]
        S = torch.cuda.Stream
        self.s_up, self.s_down = S(device=dev), S(device=dev)  # all uploads / all downloads
        self.s_cmp, self.s_dec = S(device=dev), S(device=dev)
        E = torch.cuda.Event
        names = ("up", "cmp", "down", "up2", "dec", "fetch")
        self.ev = {nm: [E(), E()] for nm in names}
        self.used = {nm: [False, False] for nm in names}
        self.nb = [0, 0]

    # -- stage helpers ------------------------------------------------------
    def _wait(self, stream, name, k):
        if self.used[name][k]:
            stream.wait_event(self.ev[name][k])

    def _record(self, stream, name, k):
        self.ev[name][k].record(stream)
        self.used[name][k] = True

    def upload(self, k: int, host_axes):
        torch = gz._torch()
        with torch.cuda.stream(self.s_up):
            self._wait(self.s_up, "cmp", k)
            for d, h in zip(self.dX[k], host_axes):
                d.copy_(h, non_blocking=True)
            self._record(self.s_up, "up", k)

    def compress(self, k: int):
        self.s_cmp.wait_event(self.ev["up"][k])
        self._wait(self.s_cmp, "down", k)
        d = self.dX[k]
        gz.compress_into(self.p, d[0], d[1], d[2] if self.dim == 3 else d[0], self.out[k], self.scr_c[k],
                         stream=self.s_cmp, sync=False)
        gz.result_post(self.scr_c[k], self.res[k], stream=self.s_cmp)
        self._record(self.s_cmp, "cmp", k)

    def stream_size(self, k: int) -> int:
        """Waits for the compress of slot k and returns its stream size.  The
        result was posted to pinned host memory by the device, so this wait
        does not queue behind the large copies of other steps."""
        self.ev["cmp"][k].synchronize()
        r = gz.Result.from_buffer_copy(self.res[k].numpy().tobytes()[:gz.ctypes.sizeof(gz.Result)])
        if r.status != 0:
            raise gz.GpzError(r.status, "SnapshotPipeline: compress failed")
        self.nb[k] = int(r.stream_bytes)
        return self.nb[k]

    def download_stream(self, k: int):
        torch = gz._torch()
        nb = self.nb[k]
        with torch.cuda.stream(self.s_down):
            self.s_down.wait_event(self.ev["cmp"][k])
            self._wait(self.s_down, "up2", k)
            self.hs[k][:nb].copy_(self.out[k][:nb], non_blocking=True)
            self._record(self.s_down, "down", k)

    def upload_stream(self, k: int):
        torch = gz._torch()
        nb = self.nb[k]
        with torch.cuda.stream(self.s_up):
            self.s_up.wait_event(self.ev["down"][k])
            self._wait(self.s_up, "dec", k)
            self.din[k][:nb].copy_(self.hs[k][:nb], non_blocking=True)
            self._record(self.s_up, "up2", k)

    def decompress(self, k: int):
        self.s_dec.wait_event(self.ev["up2"][k])
        self._wait(self.s_dec, "fetch", k)
        o = self.oX[k]
        gz.decompress_into(self.din[k], self.nb[k], self.bits, self.dim, o[0], o[1], o[2] if self.dim == 3 else o[0],
                           self.scr_d[k], stream=self.s_dec, sync=False)
        self._record(self.s_dec, "dec", k)

    def fetch(self, k: int):
        torch = gz._torch()
        with torch.cuda.stream(self.s_down):
            self.s_down.wait_event(self.ev["dec"][k])
            for h, d in zip(self.rX[k], self.oX[k]):
                h.copy_(d, non_blocking=True)
            self._record(self.s_down, "fetch", k)

    def synchronize(self):
        for s in (self.s_up, self.s_cmp, self.s_dec, self.s_down):
            s.synchronize()

    # -- the whole schedule ---------------------------------------------------
    def round_trips(self, host_axes, steps: int):
        """`steps` round trips of the snapshot `host_axes` (pinned host
        tensors): compress to a pinned host stream, decompress that stream to
        pinned host arrays.  Returns (stream bytes, host arrays) of the last
        step; the host arrays stay valid until the slot is reused."""
        if steps < 1:
            raise gz.GpzError(gz.GPZ_EINVAL, "SnapshotPipeline: steps must be >= 1")
        self.upload(0, host_axes)
        self.compress(0)
        if steps > 1:
            self.upload(1, host_axes)
        for i in range(steps):
            k = i & 1
            self.stream_size(k)
            self.download_stream(k)
            self.upload_stream(k)  # queued after the upload of snapshot i+1
            self.decompress(k)
            if i + 1 < steps:
                self.compress(k ^ 1)
            if i >= 1:
                self.fetch(k ^ 1)  # step i-1's reconstruction, behind step i's stream download
            if i + 2 < steps:
                self.upload(k, host_axes)  # snapshot i+2 into the slot compress i has released
        self.fetch((steps - 1) & 1)
        self.synchronize()
        k = (steps - 1) & 1
        return self.nb[k], self.rX[k]
