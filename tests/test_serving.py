"""Continuous-batching server: results are the same alone and in a mix, the
ring wraps correctly under a small budget, oversize events are refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _events(p2z, counts, seed, nlayer=20, B=32, masks=True):
    evs = []
    for i, n in enumerate(counts):
        cfg = p2z.make_config(bsize=B, nevts=1, event_ntrks=[n], nlayer=nlayer)
        t, h, m = p2z.generate_physics(cfg, p2z.physics_params(seed=seed + i), with_mask=True)
        if masks:
            p2z.mask_layers(m, nlayer, min_hits=5, max_hits=nlayer, drop_prob=0.1, seed=seed + 100 + i)
        evs.append((t, h, m if masks else None, n, np.zeros_like(t)))
    return evs


def test_event_alone_equals_event_in_mix(p2z, ctx):
    # the 20000-track event first, with one group in flight: the others are submitted while its
    # group (copies of ~17 MB, then the kernel) runs, so they are admitted together and mixed
    evs = _events(p2z, [20000, 3000, 50, 777, 1, 0, 4096, 1500], seed=40)
    with p2z.Server(bsize=32, nlayer=20, budget_bytes=2 << 30, max_inflight=1) as srv:
        # alone, one at a time
        alone = []
        for t, h, m, n, _ in evs:
            out = np.zeros_like(t)
            srv.wait(srv.submit(t, h, m, n, out))
            alone.append(out)
        # all at once (submitted back to back by the library's replay loop): while the first
        # group runs the others are admitted together and launched in mixed groups
        infos = srv.replay(evs, [0.0] * len(evs))
    assert max(inf.group_events for inf in infos) > 1
    for (t, h, m, n, o), a in zip(evs, alone):
        assert np.array_equal(o.view(np.uint32), a.view(np.uint32))
    # and equal to a one-event p2z_run of the same kernel arithmetic
    t, h, m, n, o = evs[0]
    cfg = p2z.make_config(bsize=32, nevts=1, event_ntrks=[n], nlayer=20, schedule="persistent")
    ref = np.empty_like(t)
    ctx.run(cfg, t, h, ref, hit_mask=m)
    assert np.array_equal(ref.view(np.uint32), o.view(np.uint32))


def test_ring_wraps_under_small_budget(p2z, ctx):
    counts = [int(x) for x in np.random.default_rng(3).integers(1, 3000, size=40)]
    evs = _events(p2z, counts, seed=90, masks=False)
    per_batch = 2 * 28 * 32 * 4 + 20 * 9 * 32 * 4 + 32 * 4
    budget = per_batch * 200          # 200 batches: far fewer than the 40 events need
    with p2z.Server(bsize=32, nlayer=20, budget_bytes=budget, max_inflight=3) as srv:
        ids = [srv.submit(t, h, m, n, o) for (t, h, m, n, o) in evs]
        infos = [srv.wait(i) for i in ids]
        assert all(i.status == p2z.OK for i in infos)
        with pytest.raises(p2z.P2zError) as e:
            big = _events(p2z, [201 * 32], seed=7, masks=False)[0]
            srv.submit(big[0], big[1], None, big[3], big[4])
        assert e.value.status == p2z.OOM
    for (t, h, m, n, o) in evs:
        cfg = p2z.make_config(bsize=32, nevts=1, event_ntrks=[n], nlayer=20)
        ref = np.empty_like(t)
        ctx.run(cfg, t, h, ref)
        assert np.array_equal(ref.view(np.uint32), o.view(np.uint32))


def test_replay_reports_latencies(p2z, ctx):
    evs = _events(p2z, [1000, 2000, 5000, 300] * 4, seed=200)
    arr = np.arange(len(evs)) * 2e-4
    with p2z.Server(bsize=32, nlayer=20, budget_bytes=1 << 30) as srv:
        infos = srv.replay(evs, arr)
    lat = np.array([i.done_s - i.submit_s for i in infos])
    assert (lat > 0).all() and (lat < 30).all()
    assert all(i.admit_s >= i.submit_s and i.launch_s >= i.admit_s and i.done_s >= i.launch_s for i in infos)
    assert sum(i.updates for i in infos) == sum(int(np.unpackbits(e[2].view(np.uint8)).sum()) for e in evs)


def test_poll_wait_timeout_and_release(p2z):
    """A request that cannot have finished (its inputs are still being
    copied) reports NOT_READY to poll and TIMEOUT to a wait that has already
    run out; waiting completes it; a reported request is released, and an
    unknown id is an error."""
    n = 300000
    cfg = p2z.make_config(bsize=32, nevts=1, event_ntrks=[n], nlayer=20)
    nb = p2z.num_batches(cfg)
    t, h, o = p2z.PinnedArray((nb, 28, 32)), p2z.PinnedArray((nb, 20, 9, 32)), p2z.PinnedArray((nb, 28, 32))
    try:
        p2z.generate_physics(cfg, out=(t.array, h.array, None))
        with p2z.Server(bsize=32, nlayer=20, budget_bytes=2 << 30) as srv:
            rid = srv.submit(t.array, h.array, None, n, o.array)
            assert srv.poll(rid) is None  # 216 MB of hits cannot have crossed the bus yet
            with pytest.raises(p2z.P2zError) as e:
                srv.wait(rid, timeout=1e-9)
            assert e.value.status == p2z.TIMEOUT
            info = srv.wait(rid, timeout=600.0)
            assert info.status == p2z.OK and info.ntrks == n and info.updates == n * 20
            assert info.submit_s <= info.admit_s <= info.launch_s <= info.done_s
            with pytest.raises(p2z.P2zError) as e:   # released once reported
                srv.poll(rid)
            assert e.value.status == p2z.BAD_ARG
            with pytest.raises(p2z.P2zError) as e:
                srv.wait(10 ** 9, timeout=1.0)
            assert e.value.status == p2z.BAD_ARG
        assert np.isfinite(o.array[:, :6, :]).all()
    finally:
        t.free(); h.free(); o.free()


SERVER_CONFIGS = [
    ("v2", 0, 0.0), ("v2", "reference_rounding", 0.0), ("v2", "accurate_trig", 0.0), ("v2", "full_hits", 0.0),
    ("v2_comp", 0, 0.0), ("3x3_f64", 0, 0.0), ("3x3_comp", 0, 0.0), ("f64", 0, 0.0),
    ("v2", 0, 100.0 / (-0.299792458 * 3.8)),
]


@pytest.mark.parametrize("update,flag,kfact", SERVER_CONFIGS)
def test_server_kinds_and_flags_match_p2z_run(p2z, ctx, update, flag, kfact):
    """Every update kind and flag the server takes (the 3-D kinds copy all 9
    hit words, the 2-D ones 6 unless P2Z_FLAG_FULL_HITS) and a field constant
    of its own: each event's result, submitted in a mix, equals a p2z_run of
    the same event with the same kind, flags and constant, bit for bit."""
    flags = {0: 0, "reference_rounding": p2z.FLAG_REFERENCE_ROUNDING, "accurate_trig": p2z.FLAG_ACCURATE_TRIG,
             "full_hits": p2z.FLAG_FULL_HITS}[flag]
    kf = float(np.float32(kfact))
    evs = _events(p2z, [2000, 31, 777, 0, 96], seed=300)
    with p2z.Server(bsize=32, nlayer=20, update=update, flags=flags, kfact=kf, budget_bytes=1 << 30,
                    max_inflight=2) as srv:
        infos = srv.replay(evs, [0.0] * len(evs))
    assert all(i.status == p2z.OK for i in infos)
    for t, h, m, n, o in evs:
        cfg = p2z.make_config(bsize=32, nevts=1, event_ntrks=[n], nlayer=20, update=update, flags=flags,
                              kfact=kf, schedule="persistent")
        ref = np.empty_like(t)
        ctx.run(cfg, t, h, ref, hit_mask=m)
        assert np.array_equal(ref.view(np.uint32), o.view(np.uint32)), (update, flag, n)
