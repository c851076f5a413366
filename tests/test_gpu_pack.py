"""p2z_pack_by_hits_device / p2z_unpack_tracks_device: a copy of an uneven
sample with every event's tracks in order of decreasing hit count, and the
way back.  Checked against a numpy restatement of the order (stable, per
event, padding last), word for word on the packed arrays, and end to end: a
run on the packed arrays, unpacked, equals the run on the caller's arrays bit
for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _expected_perm(counts, mask, B, nlayer):
    """Input slot of every packed slot: per event, real tracks by decreasing hit
    count (ties in slot order), then the event's padding slots in order."""
    perm = []
    s0 = 0
    all_ = (1 << nlayer) - 1
    for n in counts:
        ns = (int(n) + B - 1) // B * B
        slots = np.arange(s0, s0 + ns)
        real = slots[:n]
        hits = np.array([bin(int(mask[s]) & all_).count("1") for s in real], dtype=np.int64) if mask is not None \
            else np.full(len(real), nlayer)
        order = real[np.argsort(-hits, kind="stable")]
        perm.extend(order.tolist())
        perm.extend(slots[n:].tolist())
        s0 += ns
    return np.array(perm, dtype=np.int64)


@pytest.mark.parametrize("bsize", [8, 32, 64])
def test_pack_order_words_and_round_trip(p2z, ctx, bsize):
    import torch
    counts = np.array([50, 1, 0, 777, 31, 32, 33, 3000, 2], dtype=np.int64)
    cfg = p2z.make_config(bsize=bsize, nevts=len(counts), event_ntrks=counts, nlayer=20, schedule="persistent")
    t, h, m = p2z.generate_physics(cfg, with_mask=True)
    p2z.mask_layers(m, 20, min_hits=5, max_hits=20, drop_prob=0.1, seed=41)
    nb = p2z.num_batches(cfg)
    dt, dh, dm = torch.from_numpy(t).cuda(), torch.from_numpy(h).cuda(), torch.from_numpy(m.view(np.int32)).cuda()
    pt, ph, pm = torch.empty_like(dt), torch.empty_like(dh), torch.empty_like(dm)
    perm = torch.empty(2 * nb * bsize, dtype=torch.int64, device="cuda")
    ctx.pack_by_hits_device(cfg, dt, dh, pt, ph, perm, d_mask_in=dm, d_mask_out=pm)
    torch.cuda.synchronize()
    both = perm.cpu().numpy()
    got, inv = both[:nb * bsize], both[nb * bsize:]
    assert np.array_equal(got, _expected_perm(counts, m, bsize, 20))
    assert np.array_equal(inv[got], np.arange(nb * bsize))  # the second half is the inverse
    # the packed arrays are the input words of those slots
    T = p2z.tracks_to_soa(t)          # [28][nslots]
    H = p2z.hits_to_soa(h)            # [nlayer][9][nslots]
    assert np.array_equal(p2z.tracks_to_soa(pt.cpu().numpy()).view(np.uint32), T[:, got].view(np.uint32))
    assert np.array_equal(p2z.hits_to_soa(ph.cpu().numpy()).view(np.uint32), H[:, :, got].view(np.uint32))
    assert np.array_equal(pm.cpu().numpy().view(np.uint32), m[got])
    # a packed run, unpacked, gives every track its own bits
    ref = torch.empty_like(dt)
    ctx.run_device(cfg, dt, dh, ref, d_mask=dm)
    po, back = torch.empty_like(dt), torch.full_like(dt, float("nan"))
    st = ctx.run_device(cfg, pt, ph, po, d_mask=pm)
    ctx.unpack_tracks_device(cfg, perm, po, back)
    torch.cuda.synchronize()
    assert np.array_equal(back.cpu().numpy().view(np.uint32), ref.cpu().numpy().view(np.uint32))
    assert st.updates == int(sum(bin(int(x) & ((1 << 20) - 1)).count("1") for x in m))


def test_pack_without_mask_is_identity_and_refusals(p2z, ctx):
    import torch
    cfg = p2z.make_config(bsize=32, nevts=3, ntrks=640, nlayer=20)
    t, h = p2z.generate_physics(cfg)
    dt, dh = torch.from_numpy(t).cuda(), torch.from_numpy(h).cuda()
    pt, ph = torch.empty_like(dt), torch.empty_like(dh)
    perm = torch.empty(2 * 3 * 640, dtype=torch.int64, device="cuda")
    ctx.pack_by_hits_device(cfg, dt, dh, pt, ph, perm)
    torch.cuda.synchronize()
    assert np.array_equal(perm.cpu().numpy(), np.concatenate([np.arange(3 * 640)] * 2))
    assert np.array_equal(pt.cpu().numpy().view(np.uint32), t.view(np.uint32))
    for kw, status in ((dict(d_mask_in=torch.zeros(3 * 640, dtype=torch.int32, device="cuda")), p2z.BAD_ARG),
                       (dict(), p2z.BAD_ARG)):
        with pytest.raises(p2z.P2zError) as e:
            if kw:
                ctx.pack_by_hits_device(cfg, dt, dh, pt, ph, perm, **kw)   # mask in without mask out
            else:
                ctx.pack_by_hits_device(cfg, dt, dh, dt, ph, perm)         # packed copy aliases the input
        assert e.value.status == status
    cfg.layout = p2z.LAYOUT_SOA
    with pytest.raises(p2z.P2zError) as e:
        ctx.pack_by_hits_device(cfg, dt, dh, pt, ph, perm)
    assert e.value.status == p2z.UNSUPPORTED


@pytest.mark.parametrize("bsize", [16, 64])
def test_pack_every_event_size(p2z, ctx, bsize):
    """Events of every size the packing's gathers distinguish: from one batch
    to above 32768 slots (too large for shared memory, read directly), empty
    events among them; the order, the packed words and the round trip."""
    import torch
    counts = np.array([40000, 7, 20000, 0, 9000, 5000, 2100, 1500, 600, 300, 100, 1], dtype=np.int64)
    cfg = p2z.make_config(bsize=bsize, nevts=len(counts), event_ntrks=counts, nlayer=12, schedule="flat")
    t, h, m = p2z.generate_physics(cfg, with_mask=True)
    p2z.mask_layers(m, 12, min_hits=3, max_hits=12, drop_prob=0.2, seed=43)
    nb = p2z.num_batches(cfg)
    dt, dh, dm = torch.from_numpy(t).cuda(), torch.from_numpy(h).cuda(), torch.from_numpy(m.view(np.int32)).cuda()
    pt, ph, pm = torch.empty_like(dt), torch.empty_like(dh), torch.empty_like(dm)
    perm = torch.empty(2 * nb * bsize, dtype=torch.int64, device="cuda")
    ctx.pack_by_hits_device(cfg, dt, dh, pt, ph, perm, d_mask_in=dm, d_mask_out=pm)
    torch.cuda.synchronize()
    got = perm.cpu().numpy()[:nb * bsize]
    assert np.array_equal(got, _expected_perm(counts, m, bsize, 12))
    T, H = p2z.tracks_to_soa(t), p2z.hits_to_soa(h)
    assert np.array_equal(p2z.tracks_to_soa(pt.cpu().numpy()).view(np.uint32), T[:, got].view(np.uint32))
    assert np.array_equal(p2z.hits_to_soa(ph.cpu().numpy()).view(np.uint32), H[:, :, got].view(np.uint32))
    assert np.array_equal(pm.cpu().numpy().view(np.uint32), m[got])
    ref = torch.empty_like(dt)
    ctx.run_device(cfg, dt, dh, ref, d_mask=dm)
    po, back = torch.empty_like(dt), torch.full_like(dt, float("nan"))
    ctx.run_device(cfg, pt, ph, po, d_mask=pm)
    ctx.unpack_tracks_device(cfg, perm, po, back)
    torch.cuda.synchronize()
    assert np.array_equal(back.cpu().numpy().view(np.uint32), ref.cpu().numpy().view(np.uint32))
