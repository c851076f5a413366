"""p2z_run_device_noalloc: the persistent pass for callers that cannot allocate
device memory (their memory belongs to another allocator, or cudaMalloc and
cudaFree -- which can synchronise the device -- are not allowed on their
processing path).  Its scratch is a fixed array inside the library instead of
a p2z_context's allocations.

Checked through the C ABI against the existing entry point p2z_run_device on
the same inputs, on two calls in a row (the shared scratch keeps the previous
call's contents, so the second call shows that each call resets what must
start at zero).  The tolerance is the one the other GPU tests use (1e-5 on
parameters, 1e-4 on the covariance); the two are in fact the same kernel
arithmetic and must agree bit for bit.  This file is collected last so that a
run stopping at the first failure has already run every other test."""
import ctypes

import numpy as np
import pytest

from conftest import LIVE, cov_rel, par_rel

pytestmark = pytest.mark.gpu


def _noalloc(p2z, cfg, dt, dh, dm, do, stream):
    rc = p2z.lib.p2z_run_device_noalloc(ctypes.byref(cfg), dt.data_ptr(), dh.data_ptr(),
                                        None if dm is None else dm.data_ptr(), do.data_ptr(),
                                        ctypes.c_void_p(stream.cuda_stream))
    assert rc == p2z.OK, p2z.lib.p2z_last_error(None)


def _compare(p2z, a, b):
    ga, gb = p2z.tracks_to_aos(a), p2z.tracks_to_aos(b)
    assert par_rel(ga["par"], gb["par"]).max() <= 1e-5
    assert cov_rel(ga["cov"], gb["cov"])[:, LIVE].max() <= 1e-4
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("case", ["uneven_no_mask", "uniform", "uneven_with_mask"])
def test_noalloc_matches_run_device_on_two_calls(p2z, ctx, case):
    import torch
    counts = np.array([50, 1, 0, 777, 3000, 31, 64, 9000], dtype=np.int64)
    if case == "uniform":
        cfg = p2z.make_config(bsize=32, nevts=4, ntrks=960, nlayer=20)
        t, h = p2z.generate_physics(cfg)
        m = None
    else:
        cfg = p2z.make_config(bsize=32, nevts=len(counts), event_ntrks=counts, nlayer=20)
        t, h, m = p2z.generate_physics(cfg, with_mask=True)
        p2z.mask_layers(m, 20, min_hits=5, max_hits=20, drop_prob=0.1, seed=17)
        if case == "uneven_no_mask":
            m = None
    dt, dh = torch.from_numpy(t).cuda(), torch.from_numpy(h).cuda()
    dm = None if m is None else torch.from_numpy(m.view(np.int32)).cuda()
    # the existing entry point
    ref = torch.empty_like(dt)
    ctx.run_device(cfg, dt, dh, ref, d_mask=dm)
    ref = ref.cpu().numpy()
    # the allocation-free one, twice in a row into fresh outputs
    stream = torch.cuda.Stream()
    for _ in range(2):
        out = torch.full_like(dt, float("nan"))
        torch.cuda.synchronize()
        _noalloc(p2z, cfg, dt, dh, dm, out, stream)
        stream.synchronize()
        _compare(p2z, out.cpu().numpy(), ref)


def test_noalloc_rejects_runs_beyond_its_scratch(p2z):
    counts = np.full(40, 32768, dtype=np.int64)  # 1,310,720 slots > the 1,048,576-slot scratch
    cfg = p2z.make_config(bsize=32, nevts=len(counts), event_ntrks=counts, nlayer=20)
    rc = p2z.lib.p2z_run_device_noalloc(ctypes.byref(cfg), None, None, None, None, None)
    assert rc == p2z.BAD_ARG
    msg = p2z.lib.p2z_last_error(None).decode()
    assert "limits are 1048576 slots" in msg


def test_noalloc_event_limit_and_largest_event_count(p2z, ctx):
    """P2Z_NOALLOC_MAX_EVENTS + 1 events without a mask are refused; exactly
    P2Z_NOALLOC_MAX_EVENTS small events (some empty), which run the offsets
    scan at its largest, give run_device's results bit for bit."""
    import torch
    over = np.ones(65537, dtype=np.int64)
    cfg = p2z.make_config(bsize=8, nevts=len(over), event_ntrks=over, nlayer=20)
    assert p2z.lib.p2z_run_device_noalloc(ctypes.byref(cfg), None, None, None, None, None) == p2z.BAD_ARG
    assert "65536 events" in p2z.lib.p2z_last_error(None).decode()
    rng = np.random.default_rng(5)
    counts = rng.integers(0, 10, 65536).astype(np.int64)  # 0..9 tracks: 0, 8 or 16 slots per event
    cfg = p2z.make_config(bsize=8, nevts=len(counts), event_ntrks=counts, nlayer=20)
    t, h = p2z.generate_physics(cfg)
    assert p2z.num_batches(cfg) * 8 <= 1 << 20
    dt, dh = torch.from_numpy(t).cuda(), torch.from_numpy(h).cuda()
    ref = torch.empty_like(dt)
    ctx.run_device(cfg, dt, dh, ref)
    stream = torch.cuda.Stream()
    for _ in range(2):
        out = torch.full_like(dt, float("nan"))
        torch.cuda.synchronize()
        _noalloc(p2z, cfg, dt, dh, None, out, stream)
        stream.synchronize()
        _compare(p2z, out.cpu().numpy(), ref.cpu().numpy())


def test_noalloc_refuses_status_flags_and_runs_niter(p2z, ctx):
    """No status word comes back from this entry point, so the flags that
    report through one are refused; niter passes give the one-pass result."""
    import torch
    cfg = p2z.make_config(bsize=32, nevts=2, ntrks=256, nlayer=20)
    for flag in (p2z.FLAG_STRICT, p2z.FLAG_CHECK_INPUTS):
        cfg.flags = flag
        assert p2z.lib.p2z_run_device_noalloc(ctypes.byref(cfg), None, None, None, None, None) == p2z.UNSUPPORTED
    cfg.flags = 0
    t, h = p2z.generate_physics(cfg)
    dt, dh = torch.from_numpy(t).cuda(), torch.from_numpy(h).cuda()
    ref = torch.empty_like(dt)
    ctx.run_device(cfg, dt, dh, ref)
    cfg.niter = 3
    out = torch.full_like(dt, float("nan"))
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    _noalloc(p2z, cfg, dt, dh, None, out, stream)
    stream.synchronize()
    _compare(p2z, out.cpu().numpy(), ref.cpu().numpy())
