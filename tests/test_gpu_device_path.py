"""The device-resident batched decode (hvdg_decode_fields_device): the first
call of a batch shape tunes the solver tiling and captures the pipeline into a
CUDA graph, later calls replay it. Its outputs must equal those of the
host-buffer batched decode of the same fields (same tiling, same kernels),
on the capturing call and on two replays, including a replay after another
entry point has overwritten the context's tables."""
import ctypes as C

import numpy as np
import pytest

from hvdg import _cabi, api, synth

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _fields():
    fs = synth.mixed_batch(77, 6, 4, outer_range=(2, 4), cg_per_outer=20)
    return fs, [_cabi.default_geometry(f.standard) for f in fs]


def test_device_graph_path_matches_host_path():
    cfg = api.default_config(fast=0, cg_tol=1e-6, temporal_strength=-1.0)
    fs, geoms = _fields()
    n = len(fs)
    with api.Context(0) as ctx:
        host = ctx.decode_fields(
            [api.Field(f.samples, g, parity=f.parity, irls_outer=f.irls_outer,
                       cg_iterations=f.cg_iterations) for f, g in zip(fs, geoms)], cfg)
        d_in = [torch.from_numpy(f.samples.view(np.int16)).cuda() for f in fs]
        d_y = [torch.zeros((g.active_lines, g.active_width), dtype=torch.float32, device="cuda")
               for g in geoms]
        d_c = [torch.zeros((g.active_lines, g.active_width, 2), dtype=torch.float32,
                           device="cuda") for g in geoms]
        fin = (_cabi.FieldIn * n)()
        fout = (_cabi.FieldOut * n)()
        for i, f in enumerate(fs):
            fin[i].samples = d_in[i].data_ptr()
            fin[i].sample_type = _cabi.SAMPLES_U16
            fin[i].parity = f.parity
            fin[i].blanking_level = 16384.0
            fin[i].white_level = 51200.0
            fin[i].geometry = C.pointer(geoms[i])
            fin[i].irls_outer = f.irls_outer
            fin[i].cg_iterations = f.cg_iterations
            fout[i].luma = d_y[i].data_ptr()
            fout[i].chroma = d_c[i].data_ptr()
        torch.cuda.synchronize()

        def check(tag):
            for i in range(n):
                y = d_y[i].cpu().numpy()
                c = d_c[i].cpu().numpy().view(np.complex64)[..., 0]
                dy = np.abs(y - host[i].luma).max()
                dc = np.abs(c - host[i].chroma).max()
                assert dy <= 1e-5 and dc <= 1e-5, (tag, i, dy, dc)

        diag = ctx.decode_fields_device(fin, fout, n, cfg)      # capture
        assert diag.cg_iterations_run > 0
        check("capture")
        for t in d_y + d_c:
            t.zero_()
        torch.cuda.synchronize()
        d2 = ctx.decode_fields_device(fin, fout, n, cfg)        # replay
        check("replay")
        # the replayed graph records its own timing marks
        assert 0.0 < d2.ms_solver <= d2.ms_total, (d2.ms_solver, d2.ms_total)
        # a host-buffer call after a replay runs and agrees
        again = ctx.decode_fields(
            [api.Field(f.samples, g, parity=f.parity, irls_outer=f.irls_outer,
                       cg_iterations=f.cg_iterations) for f, g in zip(fs, geoms)], cfg)
        for a, b in zip(again, host):
            assert np.abs(a.luma - b.luma).max() <= 1e-5
        # another entry point reuses the arena; the next call must re-stage
        g = geoms[0]
        ctx.burst_lockin(synth.to_ire(fs[0].samples), g)
        for t in d_y + d_c:
            t.zero_()
        torch.cuda.synchronize()
        ctx.decode_fields_device(fin, fout, n, cfg)
        check("after another call")


def test_async_device_decode_on_caller_stream():
    """hvdg_decode_fields_device_async ordered against a caller stream: the
    inputs are written on that stream right before the call, the outputs are
    read on it right after, with no host synchronisation in between; results
    equal the synchronous decode, and hvdg_wait reports the status and the
    diagnostics (first call: tuning + capture, completed in the call; later
    calls: graph replays left in flight)."""
    cfg = api.default_config(fast=0, cg_tol=1e-6, temporal_strength=-1.0)
    fs, geoms = _fields()
    n = len(fs)
    with api.Context(0) as ctx:
        host = ctx.decode_fields(
            [api.Field(f.samples, g, parity=f.parity, irls_outer=f.irls_outer,
                       cg_iterations=f.cg_iterations) for f, g in zip(fs, geoms)], cfg)
        stream = torch.cuda.Stream()
        src = [torch.from_numpy(f.samples.view(np.int16)).cuda() for f in fs]
        d_in = [torch.zeros_like(t) for t in src]
        d_y = [torch.zeros((g.active_lines, g.active_width), dtype=torch.float32, device="cuda")
               for g in geoms]
        d_c = [torch.zeros((g.active_lines, g.active_width, 2), dtype=torch.float32,
                           device="cuda") for g in geoms]
        fin = (_cabi.FieldIn * n)()
        fout = (_cabi.FieldOut * n)()
        for i, f in enumerate(fs):
            fin[i].samples = d_in[i].data_ptr()
            fin[i].sample_type = _cabi.SAMPLES_U16
            fin[i].parity = f.parity
            fin[i].blanking_level = 16384.0
            fin[i].white_level = 51200.0
            fin[i].geometry = C.pointer(geoms[i])
            fin[i].irls_outer = f.irls_outer
            fin[i].cg_iterations = f.cg_iterations
            fout[i].luma = d_y[i].data_ptr()
            fout[i].chroma = d_c[i].data_ptr()
        torch.cuda.synchronize()
        for rep in range(3):
            with torch.cuda.stream(stream):
                for t in d_y + d_c + d_in:
                    t.zero_()
                for a, b in zip(d_in, src):
                    a.copy_(b)
                ctx.decode_fields_device_async(fin, fout, n, cfg, stream.cuda_stream)
                ys = [t.clone() for t in d_y]       # ordered after the decode on `stream`
                cs = [t.clone() for t in d_c]
            d = ctx.wait()
            assert d.cg_iterations_run > 0, rep
            stream.synchronize()
            for i in range(n):
                assert np.abs(ys[i].cpu().numpy() - host[i].luma).max() <= 1e-5, (rep, i)
                c = cs[i].cpu().numpy().view(np.complex64)[..., 0]
                assert np.abs(c - host[i].chroma).max() <= 1e-5, (rep, i)
        assert ctx.wait().cg_iterations_run == 0     # nothing outstanding


def test_contexts_on_concurrent_host_threads():
    """One context per host thread (the reference's one HvdEngine per
    thread, frame_bridge.h:137-140): two threads decoding different batches
    at the same time, each on its own context and stream, get exactly the
    results of decoding one after the other."""
    import threading
    cfg = api.default_config(fast=0, cg_tol=1e-6, temporal_strength=-1.0)
    batches = []
    for seed in (81, 82):
        fs = synth.mixed_batch(seed, 3, 2, outer_range=(2, 3), cg_per_outer=10)
        batches.append([api.Field(f.samples, _cabi.default_geometry(f.standard), parity=f.parity,
                                  irls_outer=f.irls_outer, cg_iterations=f.cg_iterations)
                        for f in fs])
    with api.Context(0) as c0, api.Context(0) as c1:
        seq = [c0.decode_fields(b, cfg) for b in batches]
        got = [None, None]

        def run(i, ctx):
            for _ in range(3):
                got[i] = ctx.decode_fields(batches[i], cfg)

        th = [threading.Thread(target=run, args=(i, c)) for i, c in enumerate((c0, c1))]
        for t in th:
            t.start()
        for t in th:
            t.join()
    for i in range(2):
        for a, b in zip(got[i], seq[i]):
            assert np.array_equal(a.luma, b.luma) and np.array_equal(a.chroma, b.chroma), i
