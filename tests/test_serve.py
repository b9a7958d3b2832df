"""Request server (gpz_server_*): requests submitted together and batched on
several streams give exactly the outputs of single calls; admission waits for
the device-memory budget.  CPU tests cover the C struct layouts and the
argument checks that run before any CUDA call."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import gpz_b200 as gz

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_struct_layouts_match_the_header(tmp_path):
    src = tmp_path / "sizes.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "gpz_b200.h"\n'
                   'int main(void) { printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(gpz_request), sizeof(gpz_completion), '
                   'sizeof(gpz_server_config), sizeof(gpz_server_stats), sizeof(gpz_batch_item), sizeof(gpz_dbatch_item), '
                   'offsetof(gpz_request, eb)); return 0; }\n')
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got == [ctypes.sizeof(gz.Request), ctypes.sizeof(gz.Completion), ctypes.sizeof(gz.ServerConfig),
                   ctypes.sizeof(gz.ServerStats), ctypes.sizeof(gz.BatchItem), ctypes.sizeof(gz.DBatchItem),
                   gz.Request.eb.offset]


@pytest.mark.parametrize("cfg", [dict(hbm_budget=1 << 30, streams=0, max_batch=4, workspace_bytes=0),
                                 dict(hbm_budget=1 << 30, streams=2, max_batch=0, workspace_bytes=0),
                                 dict(hbm_budget=0, streams=2, max_batch=4, workspace_bytes=0),
                                 dict(hbm_budget=1 << 20, streams=2, max_batch=4, workspace_bytes=1 << 20),
                                 dict(hbm_budget=1 << 30, streams=2, max_batch=4, workspace_bytes=0, flags=6)])
def test_server_create_rejects_bad_configs_before_touching_the_gpu(cfg):
    h = ctypes.c_void_p()
    assert gz.lib().gpz_server_create(ctypes.byref(gz.ServerConfig(**cfg)), ctypes.byref(h)) == gz.GPZ_EINVAL
    assert not h.value


# ---------------------------------------------------------------------------- GPU

def _inputs():
    import torch
    from oracle import pyoracle as po
    cases = [(1, 200_000, 3, 32, dict(rel_eb=1e-4)), (0, 50_000, 3, 64, dict(rel_eb=1e-5)),
             (2, 120_000, 2, 32, dict(eb=0.05, rel_mode=False, seg_size=8)), (1, 333, 3, 32, dict(rel_eb=1e-3)),
             (0, 1_000_000, 3, 32, dict(rel_eb=1e-4)), (1, 70_001, 2, 64, dict(rel_eb=1e-4))]
    out = []
    for i, (kind, n, dim, bits, kw) in enumerate(cases):
        dt = np.float32 if bits == 32 else np.float64
        x, y, z = (torch.from_numpy(a.copy()).cuda() for a in po.generate(kind, n, dim, 0.0, 400.0, 70 + i, dt))
        out.append((x, y, z if dim == 3 else None, kw))
    return out


def _single_compress(x, y, z, kw):
    rel = kw.get("rel_eb", 0.0)
    if kw.get("eb") is None:
        eb, _ = gz.rel_to_abs(x, y, z, rel)
        s, r = gz.compress(x, y, z, eb=eb, seg_size=kw.get("seg_size", 0), rel_mode=True, rel_eb=rel)
    else:
        s, r = gz.compress(x, y, z, eb=kw["eb"], seg_size=kw.get("seg_size", 0), rel_mode=kw.get("rel_mode", False),
                           rel_eb=rel)
    return s, r


@pytest.mark.gpu
@pytest.mark.parametrize("overlap", [False, True])
def test_requests_in_a_mix_equal_single_calls(overlap):
    """Compress and decompress requests submitted together (batched across
    three streams, run in order or concurrently) give the single-call bytes
    and reconstructions."""
    import torch
    from gpz_b200.serve import Server
    ins = _inputs()
    singles = [_single_compress(x, y, z, kw) for x, y, z, kw in ins]
    srv = Server(hbm_budget=2 << 30, streams=3, max_batch=4, overlap=overlap)
    try:
        tickets = []
        for (x, y, z, kw), (s, _) in zip(ins, singles):
            tickets.append(("c", srv.submit_compress(x, y, z, **kw)))
            tickets.append(("d", srv.submit_decompress(s)))
        for k, ((kind, t), i) in enumerate(zip(tickets, [j // 2 for j in range(len(tickets))])):
            c = srv.wait(t, timeout_ms=60_000)
            assert c.status == 0, (k, c.status)
            s, r = singles[i]
            if kind == "c":
                got = srv.stream_view(t, c)
                assert c.seg_size == r.seg_size and c.stream_bytes == r.stream_bytes
                assert torch.equal(got, s), k
            else:
                want = gz.decompress(s)
                for a, w in zip(srv.arrays_view(t, c), want):
                    assert (a is None) == (w is None)
                    if w is not None:
                        assert torch.equal(a.view(torch.uint8), w.view(torch.uint8)), k
            srv.release(t)
        st = srv.stats()
        assert st.completed == len(tickets) and st.queued == 0 and st.batches >= 2
        assert st.arena_free_bytes == st.arena_bytes - 3 * (64 << 20)
    finally:
        srv.close()


@pytest.mark.gpu
def test_admission_waits_for_the_budget():
    """With room for about two outputs, six requests still all complete, in
    order, as the caller releases earlier outputs."""
    import torch
    from gpz_b200.serve import Server
    from oracle import pyoracle as po
    n = 400_000
    x, y, z = (torch.from_numpy(a.copy()).cuda() for a in po.generate(1, n, 3, 0.0, 100.0, 9, np.float32))
    bound = gz.stream_bound(n, 3, 32)
    ws = 1 << 20
    srv = Server(hbm_budget=2 * ws + int(2.5 * bound), streams=2, max_batch=4, workspace_bytes=ws)
    try:
        ts = [srv.submit_compress(x, y, z, rel_eb=1e-4) for _ in range(6)]
        want, _ = _single_compress(x, y, z, dict(rel_eb=1e-4))
        for t in ts:
            c = srv.wait(t, timeout_ms=60_000)
            assert c.status == 0
            assert torch.equal(srv.stream_view(t, c), want)
            srv.release(t)
        assert srv.stats().batches >= 3  # never more than two outputs held at once
    finally:
        srv.close()
