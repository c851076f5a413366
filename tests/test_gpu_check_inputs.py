"""P2Z_FLAG_CHECK_INPUTS: the device scan of the input words a pass reads.

A NaN or Inf in a word the pass reads -- a floating-point track word of a slot
with a present layer, or a hit word the update kind reads on a present layer --
makes p2z_run_device return P2Z_NONFINITE_INPUT without running the pass (the
output is left as it was) and p2z_run return it after its pass.  Words the pass
does not read do not: the charge word, the 3 hit words the 2-D updates skip,
absent layers, padding slots.  On finite inputs the flag changes no output bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(p2z, nevts=2, ntrks=256, event_ntrks=None, with_mask=False):
    cfg = p2z.make_config(bsize=32, nevts=nevts, ntrks=ntrks, nlayer=20, event_ntrks=event_ntrks)
    if with_mask:
        t, h, m = p2z.generate_physics(cfg, with_mask=True)
        p2z.mask_layers(m, 20, min_hits=5, max_hits=15, drop_prob=0.2, seed=17)
        return cfg, t, h, m
    t, h = p2z.generate_physics(cfg)
    return cfg, t, h, None


def _dev(a):
    import torch
    return None if a is None else torch.from_numpy(np.ascontiguousarray(a).view(
        np.int32 if a.dtype == np.uint32 else a.dtype)).cuda()


def _run_device(p2z, ctx, cfg, t, h, m, flags):
    import torch
    cfg.flags = flags
    dt, dh, dm = _dev(t), _dev(h), _dev(m)
    out = torch.full_like(dt, 7.0)
    try:
        ctx.run_device(cfg, dt, dh, out, d_mask=dm)
        torch.cuda.synchronize()
        return p2z.OK, out.cpu().numpy()
    except p2z.P2zError as e:
        torch.cuda.synchronize()
        return e.status, out.cpu().numpy()


def test_finite_inputs_same_bits(p2z, ctx):
    cfg, t, h, _ = _case(p2z)
    st0, ref = _run_device(p2z, ctx, cfg, t, h, None, 0)
    st1, out = _run_device(p2z, ctx, cfg, t, h, None, p2z.FLAG_CHECK_INPUTS)
    assert st0 == st1 == p2z.OK
    assert np.array_equal(out.view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("where", ["track_cov", "track_par", "hit_v00_inf", "hit_x"])
def test_nonfinite_read_word_refused_before_the_pass(p2z, ctx, where):
    cfg, t, h, _ = _case(p2z)
    t, h = t.copy(), h.copy()
    if where == "track_cov":
        t[3, 6 + 14, 5] = np.nan
    elif where == "track_par":
        t[0, 3, 31] = np.nan
    elif where == "hit_v00_inf":
        h[7, 5, 3, 2] = np.inf
    else:
        h[2, 19, 0, 0] = np.nan
    st, out = _run_device(p2z, ctx, cfg, t, h, None, p2z.FLAG_CHECK_INPUTS)
    assert st == p2z.NONFINITE_INPUT
    assert (out == 7.0).all()  # the pass did not run


def test_words_the_pass_does_not_read(p2z, ctx):
    cfg, t, h, _ = _case(p2z)
    # the charge word and the hit's V20 (read by the 3-D updates only)
    t2, h2 = t.copy(), h.copy()
    t2[1, 27, 3] = np.nan   # the charge word holds an integer
    h2[4, 6, 6, 9] = np.nan
    st, _ = _run_device(p2z, ctx, cfg, t2, h2, None, p2z.FLAG_CHECK_INPUTS)
    assert st == p2z.OK
    cfg.update = p2z.UPDATE_3X3_F64
    st, _ = _run_device(p2z, ctx, cfg, t2, h2, None, p2z.FLAG_CHECK_INPUTS)
    assert st == p2z.NONFINITE_INPUT


def test_masks_absent_layers_and_padding(p2z, ctx):
    counts = np.array([50, 0, 777, 31], dtype=np.int64)
    cfg, t, h, m = _case(p2z, nevts=len(counts), event_ntrks=counts, with_mask=True)
    nb = p2z.num_batches(cfg)
    real = np.nonzero(m)[0]
    s = int(real[3])
    absent = [l for l in range(20) if not (int(m[s]) >> l) & 1]
    present = [l for l in range(20) if (int(m[s]) >> l) & 1]
    assert absent and present
    b, lane = s // 32, s % 32
    h_abs, h_pre = h.copy(), h.copy()
    h_abs[b, absent[0], 1, lane] = np.nan
    h_pre[b, present[-1], 1, lane] = np.nan
    assert _run_device(p2z, ctx, cfg, t, h_abs, m, p2z.FLAG_CHECK_INPUTS)[0] == p2z.OK
    assert _run_device(p2z, ctx, cfg, t, h_pre, m, p2z.FLAG_CHECK_INPUTS)[0] == p2z.NONFINITE_INPUT
    # uneven events without a mask: a padding slot (the last slot of event 0's second batch) is not read
    pad = 63
    assert pad >= 50 and pad < 64
    t_pad = t.copy()
    t_pad[pad // 32, 0, pad % 32] = np.nan
    st, _ = _run_device(p2z, ctx, cfg, t_pad, h, None, p2z.FLAG_CHECK_INPUTS)
    assert st == p2z.OK
    t_real = t.copy()
    t_real[1, 0, 17] = np.nan  # slot 49: event 0's last real track
    st, _ = _run_device(p2z, ctx, cfg, t_real, h, None, p2z.FLAG_CHECK_INPUTS)
    assert st == p2z.NONFINITE_INPUT
    assert nb * 32 == m.size


def test_soa_layout(p2z, ctx):
    cfg, t, h, _ = _case(p2z)
    ts, hs = p2z.tracks_to_soa(t), p2z.hits_to_soa(h)
    cfg.layout = p2z.LAYOUT_SOA
    assert _run_device(p2z, ctx, cfg, ts, hs, None, p2z.FLAG_CHECK_INPUTS)[0] == p2z.OK
    ts2 = ts.copy()
    ts2[20, 100] = np.inf
    assert _run_device(p2z, ctx, cfg, ts2, hs, None, p2z.FLAG_CHECK_INPUTS)[0] == p2z.NONFINITE_INPUT


@pytest.mark.parametrize("pinned", [False, True])
def test_host_buffers(p2z, ctx, pinned):
    """p2z_run scans each chunk after its copy: a clean call gives the device
    run's bits, a NaN makes it return P2Z_NONFINITE_INPUT (graph-recorded with
    page-locked buffers: 12288 tracks are 6 chunks)."""
    cfg, t, h, _ = _case(p2z, nevts=3, ntrks=4096)
    st0, ref = _run_device(p2z, ctx, cfg, t, h, None, 0)
    assert st0 == p2z.OK

    def host(a):
        if not pinned:
            return a.copy(), None
        pa = p2z.PinnedArray(a.shape, a.dtype)
        pa.array[...] = a
        return pa.array, pa
    cfg.flags = p2z.FLAG_CHECK_INPUTS
    (ht, pt), (hh, ph) = host(t), host(h)
    (ho, po) = host(np.zeros_like(t))
    st = ctx.run(cfg, ht, hh, ho)
    assert st.updates == 3 * 4096 * 20
    assert np.array_equal(ho.view(np.uint32), ref.view(np.uint32))
    ht[200, 10, 4] = np.nan  # a covariance word of a track in the fourth of six chunks
    with pytest.raises(p2z.P2zError) as e:
        ctx.run(cfg, ht, hh, ho)
    assert e.value.status == p2z.NONFINITE_INPUT
    ht[200, 10, 4] = t[200, 10, 4]
    ctx.run(cfg, ht, hh, ho)  # clean again: the status word was reset
    assert np.array_equal(ho.view(np.uint32), ref.view(np.uint32))
    for pa in (pt, ph, po):
        if pa is not None:
            pa.free()
