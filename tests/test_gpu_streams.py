"""Ordering of the Python binding's device calls with torch's stream.

The library's own stream is not ordered with torch's.  The binding therefore
runs a device call on torch CUDA tensors on torch's current stream (the legacy
default stream is passed as cudaStreamLegacy): the library's kernels follow the
torch work that wrote the inputs, and torch's allocator cannot hand out memory
that pending torch work still reads as an output the library then writes.
Needs a B200.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bitdiff(a, b):
    return int((a.view(np.uint32) != b.view(np.uint32)).sum())


@pytest.mark.parametrize("schedule", ["flat", "persistent"])
def test_device_call_follows_pending_torch_work(p2z, ctx, schedule):
    """Inputs written by torch work still queued behind a ~20 ms spin on
    torch's stream: the pass must see them (on the context's own stream it
    would read the zeros left before the copy).  The persistent schedule's
    graph is recorded on the context's stream and replayed on torch's."""
    import torch
    cfg = p2z.make_config(bsize=32, nevts=4, ntrks=3200, nlayer=20, schedule=schedule)
    trk, hit = p2z.generate_physics(cfg)
    src_t, src_h = torch.from_numpy(trk).cuda(), torch.from_numpy(hit).cuda()
    expect = np.empty_like(trk)
    ctx.run(p2z.make_config(bsize=32, nevts=4, ntrks=3200, nlayer=20), trk, hit, expect)
    for _ in range(2):
        dt, dh = torch.zeros_like(src_t), torch.zeros_like(src_h)
        out = torch.full_like(src_t, float("nan"))
        torch.cuda.synchronize()
        torch.cuda._sleep(40_000_000)  # a bounded spin (~20 ms) on torch's current stream
        dt.copy_(src_t)
        dh.copy_(src_h)
        st = ctx.run_device(cfg, dt, dh, out)
        assert st.updates == 4 * 3200 * 20
        assert _bitdiff(out.cpu().numpy(), expect) == 0


def test_explicit_stream_is_used_as_given(p2z, ctx):
    """An explicit torch stream (or its handle) is passed through unchanged."""
    import torch
    cfg = p2z.make_config(bsize=32, nevts=2, ntrks=1600, nlayer=20)
    trk, hit = p2z.generate_physics(cfg)
    expect = np.empty_like(trk)
    ctx.run(cfg, trk, hit, expect)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        dt, dh = torch.from_numpy(trk).cuda(), torch.from_numpy(hit).cuda()
        out = torch.empty_like(dt)
    ctx.run_device(cfg, dt, dh, out, stream=s)
    s.synchronize()
    assert _bitdiff(out.cpu().numpy(), expect) == 0
    out2 = torch.empty_like(dt)
    ctx.run_device(cfg, dt, dh, out2, stream=s.cuda_stream)
    s.synchronize()
    assert _bitdiff(out2.cpu().numpy(), expect) == 0
