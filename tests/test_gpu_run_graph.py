"""p2z_run with page-locked host buffers records its copy/kernel pipeline as a
CUDA graph on the first call and replays it while the config and buffers stay
the same (pipelines of 4 or more chunk passes or per-event launches: every
case below is that long except the short page-locked call, enqueued directly).  Checked against the same calls with P2Z_FLAG_NO_GRAPH (every copy
and kernel enqueued directly) and against p2z_run_device on the same inputs,
bit for bit: uniform and uneven runs (internal padding mask and a caller's hit
mask), the per-event schedule with and without its 10 streams, sorted windows,
the SoA layout and two threads per track; replays after the inputs' contents
change (the graph copies the buffers again, it caches no result); a new
output buffer (recorded again); and the counts the stats report."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pinned(p2z, a):
    pa = p2z.PinnedArray(a.shape, a.dtype)
    pa.array[...] = a
    return pa


def _device_ref(p2z, ctx, cfg, t, h, m):
    import torch
    dt, dh = torch.from_numpy(t).cuda(), torch.from_numpy(h).cuda()
    dm = None if m is None else torch.from_numpy(m.view(np.int32)).cuda()
    out = torch.empty_like(dt)
    ctx.run_device(cfg, dt, dh, out, d_mask=dm)
    return out.cpu().numpy()


def _same(a, b):
    assert np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


CASES = ["uniform", "uneven_internal_mask", "uneven_user_mask", "per_event", "per_event_10_streams",
         "sorted_windows", "soa", "two_threads_per_track"]


@pytest.mark.parametrize("case", CASES)
def test_run_graph_matches_direct_and_device(p2z, ctx, case):
    counts = np.array([50, 1, 0, 777, 3000, 31, 64, 4000, 2, 2100], dtype=np.int64)  # 317 batches: 4 chunks
    if case in ("uniform", "soa", "two_threads_per_track"):
        cfg = p2z.make_config(bsize=32, nevts=3, ntrks=4096, nlayer=20)
        t, h = p2z.generate_physics(cfg)
        m = None
    else:
        cfg = p2z.make_config(bsize=32, nevts=len(counts), event_ntrks=counts, nlayer=20)
        t, h, m = p2z.generate_physics(cfg, with_mask=True)
        p2z.mask_layers(m, 20, min_hits=5, max_hits=20, drop_prob=0.1, seed=31)
        if case == "uneven_internal_mask":
            m = None
    if case == "soa":
        t, h = p2z.tracks_to_soa(t), p2z.hits_to_soa(h)
        cfg.layout = p2z.LAYOUT_SOA
    if case.startswith("per_event"):
        cfg.schedule = p2z.SCHED_NAMES["per_event"]
        cfg.block_threads = 64
        if case == "per_event_10_streams":
            cfg.flags = p2z.FLAG_PER_EVENT_STREAMS
    if case == "sorted_windows":
        cfg.schedule = p2z.SCHED_NAMES["flat"]
        cfg.flags = p2z.FLAG_SORT_WINDOWS
    if case == "two_threads_per_track":
        cfg.threads_per_track = 2
    ref = _device_ref(p2z, ctx, cfg, t, h, m)
    pt, ph = _pinned(p2z, t), _pinned(p2z, h)
    pm = None if m is None else _pinned(p2z, m)
    po = p2z.PinnedArray(t.shape, t.dtype)
    mask_arr = None if pm is None else pm.array
    # recorded, then replayed
    s1 = ctx.run(cfg, pt.array, ph.array, po.array, hit_mask=mask_arr)
    _same(po.array, ref)
    po.array[...] = np.nan
    s2 = ctx.run(cfg, pt.array, ph.array, po.array, hit_mask=mask_arr)
    _same(po.array, ref)
    # the direct path reports the same work
    direct = p2z.make_config(bsize=cfg.bsize, nevts=cfg.nevts, ntrks=cfg.ntrks, nlayer=20,
                             event_ntrks=None if case in ("uniform", "soa", "two_threads_per_track") else counts,
                             schedule=cfg.schedule, block_threads=cfg.block_threads,
                             flags=cfg.flags | p2z.FLAG_NO_GRAPH, layout=cfg.layout,
                             threads_per_track=cfg.threads_per_track)
    po.array[...] = np.nan
    s3 = ctx.run(direct, pt.array, ph.array, po.array, hit_mask=mask_arr)
    _same(po.array, ref)
    for a, b in ((s1, s2), (s1, s3)):
        assert (a.launches, a.updates, a.h2d_bytes, a.d2h_bytes, a.track_slots) == \
               (b.launches, b.updates, b.h2d_bytes, b.d2h_bytes, b.track_slots)
    # new input contents in the same buffers: the replay copies them again
    if case == "uniform":
        t2, h2 = p2z.generate_physics(cfg, params=p2z.physics_params(seed=4242))
        ref2 = _device_ref(p2z, ctx, cfg, t2, h2, None)
        assert not np.array_equal(ref2.view(np.uint32), ref.view(np.uint32))
        pt.array[...] = t2
        ph.array[...] = h2
        ctx.run(cfg, pt.array, ph.array, po.array)
        _same(po.array, ref2)
        # a different output buffer: recorded again, same results
        po2 = p2z.PinnedArray(t.shape, t.dtype)
        ctx.run(cfg, pt.array, ph.array, po2.array)
        _same(po2.array, ref2)
        po2.free()
    for a in (pt, ph, po, pm):
        if a is not None:
            a.free()


def test_run_graph_pageable_short_and_inplace(p2z, ctx):
    """Pageable buffers and short pipelines take the direct path; in-place runs
    (trk_out == trk_in, page-locked) replay correctly."""
    short = p2z.make_config(bsize=32, nevts=1, ntrks=1024, nlayer=20)  # 32 batches: one chunk
    t, h = p2z.generate_physics(short)
    ref = _device_ref(p2z, ctx, short, t, h, None)
    pt, ph, po = _pinned(p2z, t), _pinned(p2z, h), p2z.PinnedArray(t.shape, t.dtype)
    for _ in range(2):
        po.array[...] = np.nan
        ctx.run(short, pt.array, ph.array, po.array)
        _same(po.array, ref)
    for a in (pt, ph, po):
        a.free()
    cfg = p2z.make_config(bsize=32, nevts=4, ntrks=2048, nlayer=20)  # 256 batches: 4 chunks
    t, h = p2z.generate_physics(cfg)
    ref = _device_ref(p2z, ctx, cfg, t, h, None)
    out = np.full_like(t, np.nan)
    ctx.run(cfg, t, h, out)
    _same(out, ref)
    pt, ph = _pinned(p2z, t), _pinned(p2z, h)
    for _ in range(2):
        pt.array[...] = t
        ctx.run(cfg, pt.array, ph.array, pt.array)
        _same(pt.array, ref)
    pt.free()
    ph.free()
