"""Array layouts (AOSOA of any bsize, SoA), device relayout and the autotuner.

The SoA layout and the bsize are storage choices only: the kernels run the
same arithmetic per track, so every layout must give the same bits per track
as the reference's AOSOA layout at bsize 32.  The relayout is checked against
a numpy restatement of the slot mapping (events padded to multiples of each
bsize), and the autotuner against its own contract (one row per measured
configuration, best = fastest, tuned defaults applied to later runs)."""
import ctypes

import numpy as np
import pytest


# ---------------------------------------------------------------------------
# host-side (no GPU)
# ---------------------------------------------------------------------------

def test_soa_numpy_round_trip(p2z):
    rng = np.random.default_rng(3)
    t = rng.standard_normal((5, 28, 16)).astype(np.float32)
    h = rng.standard_normal((5, 7, 9, 16)).astype(np.float32)
    ts, hs = p2z.tracks_to_soa(t), p2z.hits_to_soa(h)
    assert ts.shape == (28, 80) and hs.shape == (7, 9, 80)
    # element p of slot s at p*nslots + s; hit element p of layer l at (l*9 + p)*nslots + s
    s = 2 * 16 + 5
    assert ts[3, s] == t[2, 3, 5] and hs[4, 6, s] == h[2, 4, 6, 5]
    assert np.array_equal(p2z.tracks_from_soa(ts, 16), t)
    assert np.array_equal(p2z.hits_from_soa(hs, 16), h)


def test_layout_field_is_validated(p2z):
    cfg = p2z.make_config(bsize=32, nevts=2, ntrks=64, nlayer=20, layout="soa")
    assert p2z.num_batches(cfg) == 4
    cfg.layout = 7
    assert p2z.lib.p2z_num_batches(ctypes.byref(cfg)) == -1
    assert b"layout 7 unknown" in p2z.lib.p2z_last_error(None)


# ---------------------------------------------------------------------------
# numpy restatement of the relayout (slot mapping per event)
# ---------------------------------------------------------------------------

def _begins(counts, B):
    return np.concatenate([[0], np.cumsum((np.asarray(counts) + B - 1) // B * B)]).astype(np.int64)


def relayout_host(trk, hits, mask, counts, B_from, B_to):
    """AOSOA(B_from) -> AOSOA(B_to) for the same events; padding slots zero."""
    tf, hf = p2z_mod.tracks_to_soa(trk), p2z_mod.hits_to_soa(hits)
    bf, bt = _begins(counts, B_from), _begins(counts, B_to)
    src = np.concatenate([bf[e] + np.arange(n) for e, n in enumerate(counts)]).astype(np.int64)
    dst = np.concatenate([bt[e] + np.arange(n) for e, n in enumerate(counts)]).astype(np.int64)
    ns = bt[-1]
    to = np.zeros((tf.shape[0], ns), np.float32)
    ho = np.zeros((hf.shape[0], hf.shape[1], ns), np.float32)
    to[:, dst] = tf[:, src]
    ho[:, :, dst] = hf[:, :, src]
    mo = None
    if mask is not None:
        mo = np.zeros(ns, np.uint32)
        mo[dst] = mask[src]
    return p2z_mod.tracks_from_soa(to, B_to), p2z_mod.hits_from_soa(ho, B_to), mo


p2z_mod = None


@pytest.fixture(autouse=True)
def _bind(p2z):
    global p2z_mod
    p2z_mod = p2z


def test_relayout_host_restatement_is_identity_for_equal_bsize(p2z):
    counts = [33, 0, 64, 5]
    cfg = p2z.make_config(bsize=16, nevts=4, event_ntrks=counts, nlayer=4)
    t, h, m = p2z.generate_physics(cfg, with_mask=True)
    t2, h2, m2 = relayout_host(t, h, m, counts, 16, 16)
    # padding slots of the generator are not guaranteed zero; compare real slots
    # (as bit patterns: the charge word of q = -1 reads as a float NaN)
    real = np.concatenate([_begins(counts, 16)[e] + np.arange(n) for e, n in enumerate(counts)])
    assert np.array_equal(p2z.tracks_to_soa(t2)[:, real].view(np.uint32), p2z.tracks_to_soa(t)[:, real].view(np.uint32))
    assert np.array_equal(m2[real], m[real])


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------

def _physics(p2z, counts=None, nevts=4, ntrks=960, nlayer=20, masked=False, seed=11):
    if counts is None:
        cfg = p2z.make_config(bsize=32, nevts=nevts, ntrks=ntrks, nlayer=nlayer)
    else:
        cfg = p2z.make_config(bsize=32, nevts=len(counts), event_ntrks=counts, nlayer=nlayer)
    if masked:
        t, h, m = p2z.generate_physics(cfg, with_mask=True)
        p2z.mask_layers(m, nlayer, min_hits=5, max_hits=nlayer, drop_prob=0.1, seed=seed)
        return cfg, t, h, m
    t, h = p2z.generate_physics(cfg)
    return cfg, t, h, None


def _cfg_like(p2z, cfg, counts, **kw):
    base = dict(bsize=cfg.bsize, nevts=cfg.nevts, nlayer=cfg.nlayer, update=cfg.update, flags=cfg.flags)
    base.update(kw)
    if counts is None:
        return p2z.make_config(ntrks=cfg.ntrks, **base)
    return p2z.make_config(event_ntrks=counts, **base)


@pytest.mark.gpu
@pytest.mark.parametrize("update", ["v2", "3x3_f64"])
@pytest.mark.parametrize("masked", [False, True])
def test_soa_equals_aosoa_on_device(p2z, ctx, update, masked):
    import torch
    counts = [700, 31, 0, 1500, 64] if masked else None
    cfg, t, h, m = _physics(p2z, counts, masked=masked)
    cfg.update = p2z.UPDATE_NAMES[update]
    dm = None if m is None else torch.from_numpy(m.view(np.int32)).cuda()
    dt, dh = torch.from_numpy(t).cuda(), torch.from_numpy(h).cuda()
    ref = torch.empty_like(dt)
    ctx.run_device(cfg, dt, dh, ref, d_mask=dm)
    soa_cfg = _cfg_like(p2z, cfg, counts, layout="soa")
    st, sh = torch.from_numpy(p2z.tracks_to_soa(t)).cuda(), torch.from_numpy(p2z.hits_to_soa(h)).cuda()
    so = torch.empty_like(st)
    for sched in ("flat", "persistent"):
        soa_cfg.schedule = p2z.SCHED_NAMES[sched]
        so.fill_(float("nan"))
        ctx.run_device(soa_cfg, st, sh, so, d_mask=dm)
        got = p2z.tracks_from_soa(so.cpu().numpy(), 32)
        assert np.array_equal(got.view(np.uint32), ref.cpu().numpy().view(np.uint32)), sched


@pytest.mark.gpu
@pytest.mark.parametrize("update", ["v2", "3x3_f64"])
def test_soa_host_pass_equals_aosoa(p2z, ctx, update):
    """p2z_run with SoA host arrays: pitched copies of 6 (2-D updates) or all 9
    hit words per layer, chunked over slot ranges."""
    cfg, t, h, _ = _physics(p2z, nevts=8, ntrks=9600, nlayer=20)
    cfg.update = p2z.UPDATE_NAMES[update]
    out = np.empty_like(t)
    ctx.run(cfg, t, h, out)
    soa_cfg = _cfg_like(p2z, cfg, None, layout="soa")
    ts, hs = p2z.tracks_to_soa(t), p2z.hits_to_soa(h)
    so = np.full_like(ts, np.nan)
    st = ctx.run(soa_cfg, ts, hs, so)
    assert np.array_equal(p2z.tracks_from_soa(so, 32).view(np.uint32), out.view(np.uint32))
    assert st.h2d_bytes > 0 and st.d2h_bytes == t.nbytes


@pytest.mark.gpu
def test_relayout_device_matches_host_restatement(p2z, ctx):
    import torch
    counts = [100, 0, 33, 257, 8, 64]
    cfg, t, h, m = _physics(p2z, counts, nlayer=6, masked=True)
    dt, dh = torch.from_numpy(t).cuda(), torch.from_numpy(h).cuda()
    dm = torch.from_numpy(m.view(np.int32)).cuda()
    for B_to in (8, 16, 64):
        want_t, want_h, want_m = relayout_host(t, h, m, counts, 32, B_to)
        to_cfg = _cfg_like(p2z, cfg, counts, bsize=B_to)
        ot, oh = torch.full((want_t.size,), float("nan")).cuda(), torch.full((want_h.size,), float("nan")).cuda()
        om = torch.full((want_m.size,), -1, dtype=torch.int32).cuda()
        ctx.relayout_device(cfg, to_cfg, dt, dh, ot, oh, dm, om)
        assert np.array_equal(ot.cpu().numpy().view(np.uint32), want_t.reshape(-1).view(np.uint32))
        assert np.array_equal(oh.cpu().numpy().view(np.uint32), want_h.reshape(-1).view(np.uint32))
        assert np.array_equal(om.cpu().numpy().view(np.uint32), want_m)
    # AOSOA(32) -> SoA -> AOSOA(8) -> AOSOA(32) returns the input's real slots
    soa_cfg = _cfg_like(p2z, cfg, counts, layout="soa")
    b8_cfg = _cfg_like(p2z, cfg, counts, bsize=8)
    n32 = t.size
    st_, sh_ = torch.empty(n32).cuda(), torch.empty(h.size).cuda()
    ctx.relayout_device(cfg, soa_cfg, dt, dh, st_, sh_)
    w8 = relayout_host(t, h, None, counts, 32, 8)
    t8, h8 = torch.empty(w8[0].size).cuda(), torch.empty(w8[1].size).cuda()
    ctx.relayout_device(soa_cfg, b8_cfg, st_, sh_, t8, h8)
    back_t, back_h = torch.empty(n32).cuda(), torch.empty(h.size).cuda()
    ctx.relayout_device(b8_cfg, cfg, t8, h8, back_t, back_h)
    want_t, want_h, _ = relayout_host(t, h, None, counts, 32, 32)
    assert np.array_equal(back_t.cpu().numpy().view(np.uint32), want_t.reshape(-1).view(np.uint32))
    assert np.array_equal(back_h.cpu().numpy().view(np.uint32), want_h.reshape(-1).view(np.uint32))


@pytest.mark.gpu
def test_relayout_rejects_different_events(p2z, ctx):
    import torch
    a = p2z.make_config(bsize=32, nevts=2, event_ntrks=[10, 20], nlayer=4)
    b = p2z.make_config(bsize=16, nevts=2, event_ntrks=[10, 21], nlayer=4)
    x = torch.zeros(4096).cuda()
    with pytest.raises(p2z.P2zError) as e:
        ctx.relayout_device(a, b, x, x, x, x)
    assert e.value.status == p2z.BAD_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("masked", [False, True])
def test_autotune_contract(p2z, masked):
    import torch
    counts = [400, 33, 1200, 0, 97, 640, 2048, 5]
    cfg, t, h, m = _physics(p2z, counts, masked=masked)
    dt, dh = torch.from_numpy(t).cuda(), torch.from_numpy(h).cuda()
    dm = None if m is None else torch.from_numpy(m.view(np.int32)).cuda()
    with p2z.Context(0) as c:
        ref = torch.empty_like(dt)
        c.run_device(cfg, dt, dh, ref, d_mask=dm, stats=False)
        torch.cuda.synchronize()
        best, rows = c.autotune(cfg, dt, dh, d_mask=dm, reps=2)
        # bsize x layout x (flat, persistent, per-event) x threads per track {1, 2} x block,
        # masked: x window sorting {off, on} for flat and persistent,
        # + the staged schedule (one thread per track) at bsize 32 AOSOA
        per_bl = (2 * 2 + 1) * 2 * 4 if masked else 3 * 2 * 4
        assert len(rows) == 4 * 2 * per_bl + 4
        assert {r["threads_per_track"] for r in rows} == {1, 2}
        assert {r["sorted_windows"] for r in rows} == ({False, True} if masked else {False})
        assert not any(r["sorted_windows"] for r in rows if r["schedule"] in ("per_event", "staged"))
        assert {r["threads_per_track"] for r in rows if r["schedule"] == "staged"} == {1}
        assert {r["bsize"] for r in rows} == {8, 16, 32, 64}
        assert {r["layout"] for r in rows} == {"aosoa", "soa"}
        assert {r["schedule"] for r in rows} == {"flat", "persistent", "per_event", "staged"}
        assert {(r["bsize"], r["layout"]) for r in rows if r["schedule"] == "staged"} == {(32, "aosoa")}
        assert {r["block_threads"] for r in rows} == {32, 64, 128, 256}
        assert best["ms"] == min(r["ms"] for r in rows) and best["ms"] > 0
        assert all(r["updates_per_s"] > 0 for r in rows)
        # later runs with open block/schedule/threads per track at bsize 32, AOSOA use the tuned shape
        mine = min((r for r in rows if r["bsize"] == 32 and r["layout"] == "aosoa"), key=lambda r: r["ms"])
        out = torch.empty_like(dt)
        st = c.run_device(cfg, dt, dh, out, d_mask=dm)
        nonempty = sum(1 for n in counts if n > 0)
        assert st.launches == (nonempty if mine["schedule"] == "per_event" else 1)
        assert np.array_equal(out.cpu().numpy().view(np.uint32), ref.cpu().numpy().view(np.uint32))
