"""Device-side generation of the physics sample and of layer masks against
the host generator: the same per-slot double expressions, so equal except for
rare one-ulp differences where CUDA's and the C library's transcendental
functions round a double differently; layer masks (no library functions) are
bit-identical."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ulps(a, b):
    ai, bi = a.view(np.int32).astype(np.int64), b.view(np.int32).astype(np.int64)
    ai = np.where(ai < 0, -(ai & 0x7FFFFFFF), ai)
    bi = np.where(bi < 0, -(bi & 0x7FFFFFFF), bi)
    return np.abs(ai - bi)


@pytest.mark.parametrize("bsize", [8, 32])
def test_device_generator_matches_host(p2z, ctx, bsize):
    import torch
    counts = [1500, 0, 33, 4096, 7, 640, 2049]
    cfg = p2z.make_config(bsize=bsize, nevts=len(counts), event_ntrks=counts, nlayer=20)
    t, h, m = p2z.generate_physics(cfg, with_mask=True)
    dt = torch.full((t.size,), float("nan")).cuda()
    dh = torch.full((h.size,), float("nan")).cuda()
    dm = torch.full((m.size,), -1, dtype=torch.int32).cuda()
    ctx.generate_physics_device(cfg, dt, dh, dm)
    gt = dt.cpu().numpy().reshape(t.shape)
    gh = dh.cpu().numpy().reshape(h.shape)
    assert np.array_equal(dm.cpu().numpy().view(np.uint32), m)
    assert np.array_equal(gt[:, 27, :].view(np.int32), t[:, 27, :].view(np.int32))  # charges
    ut, uh = _ulps(gt[:, :27, :], t[:, :27, :]), _ulps(gh, h)
    print("words differing: tracks", int((ut > 0).sum()), "of", ut.size, "hits", int((uh > 0).sum()), "of", uh.size,
          "max ulps", int(ut.max()), int(uh.max()))
    assert ut.max() <= 2 and uh.max() <= 2
    assert (ut > 0).mean() < 1e-3 and (uh > 0).mean() < 1e-3


def test_device_mask_layers_bit_identical(p2z, ctx):
    import torch
    counts = [300, 0, 1000, 77]
    cfg = p2z.make_config(bsize=32, nevts=len(counts), event_ntrks=counts, nlayer=20)
    _, _, m = p2z.generate_physics(cfg, with_mask=True)
    dm = torch.from_numpy(m.view(np.int32).copy()).cuda()
    p2z.mask_layers(m, 20, min_hits=5, max_hits=20, drop_prob=0.1, seed=42)
    ctx.mask_layers_device(dm, m.size, 20, min_hits=5, max_hits=20, drop_prob=0.1, seed=42)
    torch.cuda.synchronize()
    assert np.array_equal(dm.cpu().numpy().view(np.uint32), m)


def test_pass_on_device_generated_input(p2z, ctx):
    """Generate on the device, run the hot path there, compare with the same
    pass on the host-generated input."""
    import torch
    from conftest import par_rel
    cfg = p2z.make_config(bsize=32, nevts=4, ntrks=2400, nlayer=20)
    t, h = p2z.generate_physics(cfg)
    dt, dh = torch.empty(t.size).cuda(), torch.empty(h.size).cuda()
    ctx.generate_physics_device(cfg, dt, dh)
    out_dev = torch.empty_like(dt)
    ctx.run_device(cfg, dt, dh, out_dev)
    out_host = torch.empty_like(dt)
    ctx.run_device(cfg, torch.from_numpy(t).cuda(), torch.from_numpy(h).cuda(), out_host)
    a = p2z.tracks_to_aos(out_dev.cpu().numpy().reshape(t.shape))
    b = p2z.tracks_to_aos(out_host.cpu().numpy().reshape(t.shape))
    assert par_rel(a["par"], b["par"]).max() <= 1e-5


def _prepare_both(p2z, ctx, seed, bsize, nevts, ntrks, smear=1e-7, cov_scale=100.0):
    import time
    import torch
    trk0, hits0 = p2z.make_atrk(*seed[0]), p2z.make_ahits(seed[1])
    t0 = time.perf_counter()
    t, h = p2z.prepare(trk0, hits0, bsize, nevts, ntrks, 20, smear=smear, cov_scale=cov_scale)
    host_s = time.perf_counter() - t0
    dt = torch.full((t.size,), float("nan")).cuda()
    dh = torch.full((h.size,), float("nan")).cuda()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.prepare_device(trk0, hits0, bsize, nevts, ntrks, 20, dt, dh, smear=smear, cov_scale=cov_scale)
    torch.cuda.synchronize()
    dev_s = time.perf_counter() - t0
    return t, h, dt.cpu().numpy().reshape(t.shape), dh.cpu().numpy().reshape(h.shape), host_s, dev_s


@pytest.mark.parametrize("bsize", [8, 16, 32, 64])
def test_prepare_device_equals_prepare(p2z, ctx, kat_seed, bsize):
    """The reference's prepareTracks / prepareHits on the device: the words of
    p2z_prepare (itself bit-exact with the reference's own functions)."""
    t, h, gt, gh, _, _ = _prepare_both(p2z, ctx, kat_seed, bsize, 2, 128)
    assert np.array_equal(t.view(np.uint32), gt.view(np.uint32))
    assert np.array_equal(h.view(np.uint32), gh.view(np.uint32))


@pytest.mark.parametrize("case", ["known_answer", "single_seed"])
def test_prepare_device_full_size(p2z, ctx, kat_seed, readme_seed, case):
    """The known-answer workload (100 x 9600, smear 1e-7, covariances x100)
    and the single-seed one (10 x 9600, smear 1e-5, covariances as given),
    word for word, with the host and device setup times printed."""
    if case == "known_answer":
        t, h, gt, gh, hs, ds = _prepare_both(p2z, ctx, kat_seed, 32, 100, 9600)
    else:
        t, h, gt, gh, hs, ds = _prepare_both(p2z, ctx, readme_seed, 32, 10, 9600, smear=1e-5, cov_scale=1.0)
    print(f"{case}: host p2z_prepare {hs:.3f} s, p2z_prepare_device {ds:.4f} s ({hs / ds:.0f}x)")
    assert int((t.view(np.uint32) != gt.view(np.uint32)).sum()) == 0
    assert int((h.view(np.uint32) != gh.view(np.uint32)).sum()) == 0
