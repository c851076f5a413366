"""The validation block reduced on the GPU (p2z_validate_device) against the
host block (p2z_validate), on the reference's own outputs and on the physics
workload after a pass: identical counts, sums within 1e-12 relative (same
summands, different summation order), and the same printed text."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ["avgx", "avgy", "avgz", "avgdx", "avgdy", "avgdz", "avgpt", "avgphi", "avgtheta",
          "stdx", "stdy", "stdz", "stddx", "stddy", "stddz"]


def _close(a, b, rel=1e-12):
    return abs(a - b) <= rel * max(abs(a), abs(b), 1e-300) or a == b


def _compare(p2z, v_dev, v_host):
    assert (v_dev.nnans, v_dev.nfail, v_dev.ngood) == (v_host.nnans, v_host.nfail, v_host.ngood)
    for f in FIELDS:
        a, b = getattr(v_dev, f), getattr(v_host, f)
        # the std fields are sqrtf of the float-rounded mean square, as in the reference
        assert _close(a, b, 1e-12 if f.startswith("avg") else 1e-6), (f, a, b)


def test_device_block_on_reference_outputs(p2z, ctx, kat_seed):
    import torch
    import pathlib
    gold = np.load(pathlib.Path(__file__).parent / "golden" / "ref_kat_small.npz")["out_fma"]
    hit_last = kat_seed[1][19][0]
    v_host = p2z.validate(gold, 32, 2, 128, hit_last)
    v_dev = ctx.validate_device(torch.from_numpy(gold).cuda(), 32, 2, 128, hit_last)
    _compare(p2z, v_dev, v_host)
    assert v_dev.ngood == 256


@pytest.mark.parametrize("bsize", [16, 32])
def test_device_block_after_a_pass(p2z, ctx, bsize):
    import torch
    cfg = p2z.make_config(bsize=bsize, nevts=6, ntrks=4800, nlayer=20)
    t, h = p2z.generate_physics(cfg)
    dt, dh = torch.from_numpy(t).cuda(), torch.from_numpy(h).cuda()
    do = torch.empty_like(dt)
    ctx.run_device(cfg, dt, dh, do)
    out = do.cpu().numpy()
    # move the angles into the reference's fixed window (phi ~ 1.3, theta ~ 2.8;
    # the physics sample is forward, theta ~ 0.2-0.4) and pick a window point
    # inside the sample, so that the block has good and failed tracks alike
    out[:, 0, :] += 50.0
    out[:, 1, :] += 50.0
    out[:, 4, :] = 1.3 + 0.5 * np.sin(out[:, 4, :])
    out[:, 5, :] = 2.5 + out[:, 5, :]
    out[:, 4, ::7] = 10.0  # outside the window: failed tracks
    hit_last = [50.0, 50.0, float(np.median(out[:, 2, :]))]
    out[0, 0, 3] = np.nan
    do.copy_(torch.from_numpy(out))
    v_host = p2z.validate(out, bsize, 6, 4800, hit_last)
    v_dev = ctx.validate_device(do, bsize, 6, 4800, hit_last)
    _compare(p2z, v_dev, v_host)
    assert v_dev.nnans == 1 and v_dev.ngood > 1000 and v_dev.nfail > 1000
    # the per-shard form: pass 1 then pass 2 on the global means
    p1 = ctx.validate_partial_device(do, bsize, 6, 4800, hit_last)
    means = np.array(p1.sum[:6]) / p1.ngood
    p2 = ctx.validate_partial_device(do, bsize, 6, 4800, hit_last, means=means)
    assert p1.ngood == v_host.ngood and p2.ngood == v_host.ngood
    assert all(_close(p1.sum[i], getattr(v_host, FIELDS[i]) * v_host.ngood, 1e-12) for i in range(9))


def test_device_block_rejects_bad_sizes(p2z, ctx):
    import torch
    x = torch.zeros(28 * 32).cuda()
    with pytest.raises(p2z.P2zError) as e:
        ctx.validate_device(x, 32, 1, 33, [1.0, 1.0, 1.0])
    assert e.value.status == p2z.BAD_ARG
