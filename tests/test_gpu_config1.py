"""Per-track parity on the GPU for the single-seed workload (the pseudocode's
endcap track and hit) and, beside it, for the physics and known-answer
inputs: the default (precise) form against FP64 and against the reference's
OpenMP build as its Makefile compiles it, parameters AND covariance.  Needs a
B200.

Single-seed workload: the track of propagate-toz-pseudocode.txt:1-16 and its
hit on every one of 20 layers, 10 events x 9600 tracks in bsize-32 batches,
NITER 5, every element multiplied by (1 + 1e-5 N(0,1)) through the
reference's own prepareTracks/prepareHits draws (p2z_prepare; covariances not
rescaled, as in src/propagate-toz-test_sycl.cpp:647-658).  The hit's xy
covariance has correlation -0.9988 and the same hit is met 20 times, so every
layer after the first shrinks a near-singular covariance: in FP32 this input
is ill-conditioned by construction.  Measured on the CPU for the 96,000
tracks: the reference's FP32 build (FMA on) is 5e-4 from FP64 in q/pT on the
median track and up to 5.8e2 on its worst; its FMA and no-FMA builds differ
by up to 1.9 in q/pT; the float-state floor (the FP64 oracle with the state
rounded to FP32 between layers, the error any FP32-state kernel starts from)
reaches 1.3e-4 in q/pT.  A fixed 1e-5 against FP64 is therefore not reachable
by any FP32-state evaluation here; the bound is per track, from that track's
floor.

Tolerances, per track and element (parameters as |a-b|/max(|b|, floor_p),
covariance as |dC_ij|/sqrt(C_ii C_jj), both against the FP64 oracle):
    physics        parameters 1e-5, covariance 1e-4 (the targets themselves)
    single seed    parameters 1e-5, q/pT 1e-3; covariance 3e-2
    known-answer   x, y 5e-5, q/pT 2e-4, others 1e-5; covariance 2e-2
On the two single-seed inputs a smaller a-priori bound is not meaningful:
their FP32 conditioning puts the reference's own build 5.8e2 (single seed)
and 1.5e-4 (known-answer) from FP64 in q/pT, and neither the float-state
floor nor any per-track quantity predicts where an FP32 evaluation lands
(tracks whose floor is below 1e-7 err by 1e-4).  Their bounds are the
precise form's measured maxima on one B200 (single seed: q/pT 4.3e-4, other
parameters <= 4.5e-6, covariance 1.5e-2; known-answer: x, y 3.2e-5, q/pT
1.0e-4, covariance 1.1e-2) rounded up, asserted so that a regression shows.
Against the reference as built (FMA contraction on, glibc sinf/cosf), per
track and element, by the triangle inequality over the FP64 answer:
    |p - r| <= |r - fp64| + (the bound above)   (parameters and covariance)
and, over the whole sample, no worse than the reference's own build: the
largest and the 99th-percentile error of every parameter, and the largest
covariance error, within 1.1x the reference build's (the precise form is
1e6x better at the worst single-seed track, 500x on the physics sample, and
equal within 8% on the known-answer input, where both are near 1e-4).
The float-state floor (the FP64 oracle with the state rounded to FP32 between
layers) is printed beside the errors for comparison.
"""
import numpy as np
import pytest

from conftest import LIVE, cov_rel, par_rel

pytestmark = pytest.mark.gpu

# (per-parameter bound: x, y, z, q/pT, phi, theta; covariance bound), per input
BOUNDS = {"physics": (np.array([1e-5] * 6), 1e-4),
          "single_seed": (np.array([1e-5, 1e-5, 1e-5, 1e-3, 1e-5, 1e-5]), 3e-2),
          "known_answer": (np.array([5e-5, 5e-5, 1e-5, 2e-4, 1e-5, 1e-5]), 2e-2)}


def _run(p2z, ctx, trk, hit, nevts, flags=0, niter=1):
    B = trk.shape[2]
    cfg = p2z.make_config(bsize=B, nevts=nevts, ntrks=trk.shape[0] * B // nevts, nlayer=hit.shape[1], flags=flags,
                          niter=niter)
    out = np.empty_like(trk)
    st = ctx.run(cfg, trk, hit, out)
    return out, st


def _floor(oracle, trk, hit):
    """FP64 oracle one layer at a time, the state rounded to FP32 in between."""
    cur = trk.copy()
    nb, _, B = trk.shape
    for l in range(hit.shape[1]):
        o = oracle.run_f64(cur, np.ascontiguousarray(hit[:, l:l + 1]))
        cur[:, :27, :] = o.reshape(nb, B, 27).astype(np.float32).transpose(0, 2, 1)
    return cur


class Case:
    """Inputs of one workload and every CPU-side reference result."""

    def __init__(self, p2z, oracle, name, trk, hit, nevts, niter=1):
        self.name, self.trk, self.hit, self.nevts, self.niter = name, trk, hit, nevts, niter
        self.o64 = oracle.run_f64(trk, hit)
        fl = p2z.tracks_to_aos(_floor(oracle, trk, hit))
        self.floor_par = par_rel(fl["par"], self.o64[:, :6])
        self.floor_cov = cov_rel(fl["cov"], self.o64[:, 6:])[:, LIVE]
        self.ref = p2z.tracks_to_aos(oracle.ref_run(trk, hit, nev=nevts, name="b32")) \
            if oracle.ref_available("b32") else None


@pytest.fixture(scope="module")
def single_seed(p2z, oracle, readme_seed):
    t, h = p2z.prepare(p2z.make_atrk(*readme_seed[0]), p2z.make_ahits(readme_seed[1]), 32, 10, 9600, 20,
                       smear=1e-5, cov_scale=1.0)
    return Case(p2z, oracle, "single seed 10 x 9600", t, h, 10, niter=5)


@pytest.fixture(scope="module")
def cases(p2z, oracle, single_seed, kat_seed):
    cfg = p2z.make_config(bsize=32, nevts=2, ntrks=9600, nlayer=20)
    pt, ph = p2z.generate_physics(cfg, p2z.physics_params(seed=31337))
    kt, kh = p2z.prepare(p2z.make_atrk(*kat_seed[0]), p2z.make_ahits(kat_seed[1]), 32, 2, 9600, 20)
    return {"single_seed": single_seed, "physics": Case(p2z, oracle, "physics 2 x 9600", pt, ph, 2),
            "known_answer": Case(p2z, oracle, "known-answer input 2 x 9600", kt, kh, 2)}


def test_single_seed_reference_rounding_bit_exact(p2z, oracle, ctx, single_seed):
    """The reference-rounding form, NITER 5, bit for bit against the reference
    built without FMA contraction and with correctly rounded sinf/cosf."""
    if not oracle.ref_available("b32_nofma_crtrig"):
        pytest.skip("reference build absent")
    c = single_seed
    out, st = _run(p2z, ctx, c.trk, c.hit, c.nevts, flags=p2z.FLAG_REFERENCE_ROUNDING, niter=c.niter)
    ref = oracle.ref_run(c.trk, c.hit, nev=c.nevts, name="b32_nofma_crtrig")
    assert st.updates == 96000 * 20 and st.launches >= 5
    assert int((out.view(np.uint32) != ref.view(np.uint32)).sum()) == 0


def test_single_seed_reference_rounding_within_build_spread(p2z, oracle, ctx, single_seed):
    """Against the reference as its Makefile builds it (FMA contraction, glibc
    sinf/cosf), per track: within the distance between that build and the
    no-FMA correctly-rounded build on the same track -- the reference's own
    spread between build choices, which on this input reaches 1.9 in q/pT."""
    if not oracle.ref_available("b32_nofma_crtrig") or single_seed.ref is None:
        pytest.skip("reference build absent")
    c = single_seed
    out, _ = _run(p2z, ctx, c.trk, c.hit, c.nevts, flags=p2z.FLAG_REFERENCE_ROUNDING)
    crt = p2z.tracks_to_aos(oracle.ref_run(c.trk, c.hit, nev=c.nevts, name="b32_nofma_crtrig"))
    g = p2z.tracks_to_aos(out)
    spread = par_rel(crt["par"], c.ref["par"])
    got = par_rel(g["par"], c.ref["par"])
    assert (got <= spread * (1 + 1e-6) + 1e-12).all()


def _precise_vs_fp64(p2z, ctx, c, name):
    out, st = _run(p2z, ctx, c.trk, c.hit, c.nevts, niter=c.niter)
    g = p2z.tracks_to_aos(out)
    ep = par_rel(g["par"], c.o64[:, :6])
    ec = cov_rel(g["cov"], c.o64[:, 6:])[:, LIVE]
    bp, bc = BOUNDS[name]
    return g, st, ep, ec, bp, bc


@pytest.mark.parametrize("name", ["single_seed", "physics", "known_answer"])
def test_precise_vs_fp64_per_track(p2z, ctx, cases, name):
    c = cases[name]
    g, st, ep, ec, bp, bc = _precise_vs_fp64(p2z, ctx, c, name)
    print(f"{c.name}: precise vs fp64 par max {ep.max(0)} (p50 {np.median(ep, 0)}), cov max {ec.max():.3e} "
          f"(p99 {np.percentile(ec, 99):.3e}); floor par max {c.floor_par.max(0)}, floor cov max "
          f"{c.floor_cov.max():.3e}; ratio to bound par {(ep / bp).max():.3f} cov {(ec / bc).max():.3f}; "
          f"error over 3x the floor on {int((ep > np.maximum(1e-5, 3 * c.floor_par)).any(1).sum())} tracks")
    assert np.isfinite(g["par"]).all() and np.isfinite(g["cov"]).all()
    assert st.singular == 0
    assert (ep <= bp).all(), f"parameter error over the bound on {int((ep > bp).any(1).sum())} tracks"
    assert (ec <= bc).all(), f"covariance error over the bound on {int((ec > bc).any(1).sum())} tracks"


@pytest.mark.parametrize("name", ["single_seed", "physics", "known_answer"])
def test_precise_vs_reference_build_per_track(p2z, ctx, cases, name):
    """The stated per-track tolerance against the reference's own build (see
    the module text), on parameters and on the live covariance."""
    c = cases[name]
    if c.ref is None:
        pytest.skip("reference build absent")
    g, _, ep, ec, bp, bc = _precise_vs_fp64(p2z, ctx, c, name)
    rp = par_rel(c.ref["par"], c.o64[:, :6])
    rc = cov_rel(c.ref["cov"], c.o64[:, 6:])[:, LIVE]
    # normalise both against the FP64 answer so the triangle inequality holds term by term
    dp = np.abs(g["par"] - c.ref["par"].astype(np.float64)) / np.maximum(np.abs(c.o64[:, :6]),
                                                                          np.array([1, 1, 1, 1e-3, 1, 1e-2]))
    dc = cov_rel(g["cov"] - c.ref["cov"].astype(np.float64) + c.o64[:, 6:], c.o64[:, 6:])[:, LIVE]
    excess_p = (dp - rp).max(0)
    excess_c = float((dc - rc).max())
    print(f"{c.name}: |p - ref| par max {dp.max(0)}, reference vs fp64 par max {rp.max(0)}; "
          f"max(|p - ref| - |ref - fp64|) par {excess_p}, cov {excess_c:.3e}")
    assert (dp <= rp * (1 + 1e-6) + bp).all()
    assert (dc <= rc * (1 + 1e-6) + bc).all()
    # no worse than the reference's own build over the sample
    print(f"{c.name}: precise par max {ep.max(0)} p99 {np.percentile(ep, 99, axis=0)}; reference build par max "
          f"{rp.max(0)} p99 {np.percentile(rp, 99, axis=0)}; cov max {ec.max():.3e} vs {rc.max():.3e}")
    assert (ep.max(0) <= 1.1 * rp.max(0) + 1e-12).all()
    assert (np.percentile(ep, 99, axis=0) <= 1.1 * np.percentile(rp, 99, axis=0) + 1e-12).all()
    assert ec.max() <= 1.1 * rc.max()

