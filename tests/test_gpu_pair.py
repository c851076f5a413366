"""Two threads per track (p2z_config.threads_per_track = 2).

Lanes 2i and 2i+1 of a warp hold the same track; each evaluates one row of
every packed pair of the covariance propagation and takes the other row from
its partner lane by a shuffle, and both evaluate the rest of the step.  Every
output element goes through the same roundings as with one thread per track,
so the two forms must agree bit for bit: on every AOSOA bsize and SoA, the
flat and persistent schedules, masked (uneven) runs including the per-event
schedule and sorted windows, the accurate-trigonometry flag and the
ill-conditioned known-answer input (whose first updates take the Joseph
form and whose direction offsets leave their series' range)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(p2z, ctx, cfg, t, h, m=None, **kw):
    import torch
    for k, v in kw.items():
        setattr(cfg, k, p2z.SCHED_NAMES[v] if k == "schedule" else v)
    dt, dh = torch.from_numpy(t).cuda(), torch.from_numpy(h).cuda()
    dm = None if m is None else torch.from_numpy(m.view(np.int32)).cuda()
    out = torch.full_like(dt, float("nan"))
    st = ctx.run_device(cfg, dt, dh, out, d_mask=dm)
    return out.cpu().numpy(), st


def _same(a, b):
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("schedule", ["flat", "persistent"])
@pytest.mark.parametrize("layout", ["b8", "b16", "b32", "b64", "soa"])
def test_pair_bitwise_uniform(p2z, ctx, layout, schedule):
    B = 32 if layout == "soa" else int(layout[1:])
    cfg = p2z.make_config(bsize=B, nevts=3, ntrks=640, nlayer=20)
    t, h = p2z.generate_physics(cfg)
    if layout == "soa":
        t, h = p2z.tracks_to_soa(t), p2z.hits_to_soa(h)
        cfg.layout = p2z.LAYOUT_SOA
    ref, _ = _run(p2z, ctx, cfg, t, h, schedule="flat", block_threads=128, threads_per_track=1)
    for block in (32, 64, 256):
        out, st = _run(p2z, ctx, cfg, t, h, schedule=schedule, block_threads=block, threads_per_track=2)
        assert st.updates == 3 * 640 * 20
        _same(out, ref)


@pytest.mark.parametrize("schedule", ["flat", "persistent", "per_event"])
def test_pair_bitwise_uneven_masked(p2z, ctx, schedule):
    counts = np.array([50, 1, 0, 777, 3000, 31, 64, 9000, 2], dtype=np.int64)
    cfg = p2z.make_config(bsize=32, nevts=len(counts), event_ntrks=counts, nlayer=20)
    t, h, m = p2z.generate_physics(cfg, with_mask=True)
    p2z.mask_layers(m, 20, min_hits=5, max_hits=20, drop_prob=0.1, seed=23)
    ref, st1 = _run(p2z, ctx, cfg, t, h, m, schedule="flat", block_threads=128, threads_per_track=1)
    out, st2 = _run(p2z, ctx, cfg, t, h, m, schedule=schedule, block_threads=64, threads_per_track=2)
    assert st1.updates == st2.updates > 0
    _same(out, ref)
    if schedule != "per_event":
        cfg.flags = p2z.FLAG_SORT_WINDOWS
        out, _ = _run(p2z, ctx, cfg, t, h, m, schedule=schedule, block_threads=64, threads_per_track=2)
        _same(out, ref)


def test_pair_bitwise_accurate_trig_and_known_answer(p2z, ctx, kat_seed):
    cfg = p2z.make_config(bsize=32, nevts=2, ntrks=512, nlayer=20, flags=p2z.FLAG_ACCURATE_TRIG)
    t, h = p2z.generate_physics(cfg)
    ref, _ = _run(p2z, ctx, cfg, t, h, schedule="flat", block_threads=128, threads_per_track=1)
    out, _ = _run(p2z, ctx, cfg, t, h, schedule="flat", block_threads=128, threads_per_track=2)
    _same(out, ref)
    (par, cov, q), hits = kat_seed
    t, h = p2z.prepare(p2z.make_atrk(par, cov, q), p2z.make_ahits(hits), 32, 4, 9600, 20)
    cfg = p2z.make_config(bsize=32, nevts=4, ntrks=9600, nlayer=20)
    ref, _ = _run(p2z, ctx, cfg, t, h, schedule="flat", block_threads=128, threads_per_track=1)
    out, _ = _run(p2z, ctx, cfg, t, h, schedule="flat", block_threads=128, threads_per_track=2)
    _same(out, ref)


def test_pair_refusals(p2z, ctx):
    """threads_per_track outside {0, 1, 2}, 2 with an update kind or rounding
    that has no two-lane form, and 2 with the staged schedule are refused
    with P2Z_UNSUPPORTED before anything runs."""
    import torch
    cfg0 = p2z.make_config(bsize=32, nevts=1, ntrks=64, nlayer=20)
    nb = p2z.num_batches(cfg0)
    t = torch.zeros(nb * p2z.trk_words(32)).cuda()
    h = torch.zeros(nb * 20 * p2z.hit_words(32)).cuda()
    cases = [dict(threads_per_track=4), dict(threads_per_track=-1),
             dict(threads_per_track=2, update=p2z.UPDATE_NAMES["3x3_f64"]),
             dict(threads_per_track=2, flags=p2z.FLAG_REFERENCE_ROUNDING),
             dict(threads_per_track=2, schedule=p2z.SCHED_NAMES["staged"])]
    for kw in cases:
        cfg = p2z.make_config(bsize=32, nevts=1, ntrks=64, nlayer=20)
        for k, v in kw.items():
            setattr(cfg, k, v)
        with pytest.raises(p2z.P2zError) as e:
            ctx.run_device(cfg, t, h, torch.empty_like(t))
        assert e.value.status == p2z.UNSUPPORTED, kw
        assert "one thread per track" in str(e.value) or "threads_per_track" in str(e.value)


@pytest.mark.parametrize("layout", ["b8", "b64", "soa"])
def test_pair_and_sorted_windows_every_layout(p2z, ctx, layout):
    """Two threads per track and sorted windows together and apart, flat and
    persistent, on the bsizes and the layout the other tests use least:
    every combination gives the one-thread, stored-order bits."""
    counts = np.array([300, 0, 65, 1, 1000, 129], dtype=np.int64)
    B = 32 if layout == "soa" else int(layout[1:])
    cfg = p2z.make_config(bsize=B, nevts=len(counts), event_ntrks=counts, nlayer=20)
    t, h, m = p2z.generate_physics(cfg, with_mask=True)
    p2z.mask_layers(m, 20, min_hits=3, max_hits=20, drop_prob=0.2, seed=61)
    if layout == "soa":
        t, h = p2z.tracks_to_soa(t), p2z.hits_to_soa(h)
        cfg.layout = p2z.LAYOUT_SOA
    ref, _ = _run(p2z, ctx, cfg, t, h, m, schedule="flat", block_threads=64, threads_per_track=1, flags=0)
    for sched in ("flat", "persistent"):
        for tpt in (1, 2):
            for flags in (0, p2z.FLAG_SORT_WINDOWS):
                out, _ = _run(p2z, ctx, cfg, t, h, m, schedule=sched, block_threads=128, threads_per_track=tpt,
                              flags=flags)
                _same(out, ref)


def test_pair_with_32_layers(p2z, ctx):
    """Every mask bit, bit 31 included, with two threads per track."""
    cfg = p2z.make_config(bsize=32, nevts=2, ntrks=320, nlayer=32)
    t, h, m = p2z.generate_physics(cfg, with_mask=True)
    p2z.mask_layers(m, 32, min_hits=5, max_hits=32, drop_prob=0.1, seed=3)
    ref, _ = _run(p2z, ctx, cfg, t, h, m, schedule="flat", block_threads=64, threads_per_track=1)
    out, _ = _run(p2z, ctx, cfg, t, h, m, schedule="persistent", block_threads=64, threads_per_track=2)
    _same(out, ref)
