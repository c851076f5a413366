"""The benchmark's reference arm (CPU): it times the reference's own OpenMP hot
loop on the same physics sample as the GPU arm, describes the same workload in
the same `config` object, and loads nothing of the product library."""
import json
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT


@pytest.mark.parametrize("bsize,nevts,ntrks", [(32, 2, 9600), (8, 3, 64), (64, 1, 128)])
def test_oracle_physics_sample_equals_library_generator(p2z, oracle, bsize, nevts, ntrks):
    """The oracle's restatement of the physics generator (the reference arm's
    inputs) equals p2z_generate_physics word for word."""
    t, h = oracle.physics(bsize, nevts, ntrks, 20, seed=77)
    cfg = p2z.make_config(bsize=bsize, nevts=nevts, ntrks=ntrks, nlayer=20)
    t2, h2 = p2z.generate_physics(cfg, p2z.physics_params(seed=77))
    assert np.array_equal(t.view(np.uint32), t2.view(np.uint32))
    assert np.array_equal(h.view(np.uint32), h2.view(np.uint32))


_ARM = r"""
import json, runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "3", "--ref-events", "2"]
try:
    runpy.run_path("bench.py", run_name="__main__")
except SystemExit as e:
    assert not e.code, e.code
maps = open("/proc/self/maps").read()
libs = sorted({l.split()[-1] for l in maps.splitlines() if l.split()[-1].endswith(".so") or ".so." in l.split()[-1]})
print("LIBS " + json.dumps([x for x in libs if "/repo" in x or "p2z" in x or "oracle" in x]))
"""


def test_reference_arm_loads_no_product_library_and_shares_the_config(oracle):
    if not oracle.ref_available("b32"):
        pytest.skip("reference build absent")
    r = subprocess.run([sys.executable, "-c", _ARM], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.splitlines()
    line = json.loads(next(l for l in lines if l.startswith("{")))
    libs = json.loads(next(l for l in lines if l.startswith("LIBS "))[5:])
    assert not [x for x in libs if "p2z-tests_b200" in x or x.endswith("/libp2z.so")], libs
    assert all("/oracle/" in x for x in libs), libs
    assert any("oracle/_ref" in x for x in libs), libs
    assert line["impl"] == "reference" and line["unit"] == "updates/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference"
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    # the GPU arm builds its config with the same function and arguments
    sys.path.insert(0, str(ROOT))
    import importlib
    bench = importlib.import_module("bench")
    assert line["config"] == bench.workload_config(1000, 1)


def _bench_module():
    import importlib.util
    spec = importlib.util.spec_from_file_location("p2z_bench_helpers", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_window_utilisation_and_tune_summary():
    """The bench's lane-utilisation count for sorted windows and its summary of
    an autotune sweep, on inputs whose answers are known."""
    import torch
    bench = _bench_module()
    # 64 slots: window 1 holds 32 tracks of 20 hits and 32 of 4; sorted per 64-slot window the
    # two warps take 20 and 4 steps (all lanes busy); per 32-slot window (no reordering across
    # warps) each warp takes 20 steps for 16 x 20 + 16 x 4 hits
    hits = [20, 4] * 32
    mask = torch.tensor([(1 << h) - 1 for h in hits], dtype=torch.int64).to(torch.int32)
    assert bench.window_util(mask, 64) == pytest.approx(1.0)
    assert bench.window_util(mask, 32) == pytest.approx((16 * 20 + 16 * 4) / (32 * 20))
    rows = [dict(bsize=b, layout=l, schedule=s, block_threads=32, threads_per_track=t, sorted_windows=w,
                 ms=1.0 + 0.1 * b + (0.5 if l == "soa" else 0) + t + (0 if w else 0.05), updates_per_s=1.0)
            for b in (8, 32) for l in ("aosoa", "soa") for s in ("flat", "persistent") for t in (1, 2)
            for w in (False, True)]
    best = min(rows, key=lambda r: r["ms"])
    out = bench.tune_summary(best, rows, 1.5)
    assert out["configurations"] == len(rows) and out["best"] is best
    assert out["best_bsize32_aosoa"]["bsize"] == 32 and out["best_bsize32_aosoa"]["layout"] == "aosoa"
    assert set(out["best_per_sorted_windows"]) == {"False", "True"}
    assert out["best_per_threads_per_track"]["1"]["ms"] < out["best_per_threads_per_track"]["2"]["ms"]


def test_clock_record_window():
    """The bench's clock record: the samples inside the timed region, their
    median and every throttle reason among them; with none inside (a region
    shorter than the sampler's period) the samples within 0.25 s of it."""
    bench = _bench_module()
    c = bench.ClockSampler(0)
    c.sm_max = 1965.0
    c.samples = [(0.90, 1500.0, 0x4), (1.00, 1965.0, 0), (1.01, 1965.0, 0x4), (1.02, 1950.0, 0), (1.60, 1200.0, 0x8)]
    r = c.stop(0.995, 1.025)
    assert (r["sm_mhz"], r["samples"], r["reasons"], r["window"]) == (1965.0, 3, ["sw_power_cap"], "timed region")
    c = bench.ClockSampler(0)
    c.samples = [(0.90, 1900.0, 0), (1.20, 1965.0, 0x8), (2.00, 1000.0, 0x40)]
    r = c.stop(1.05, 1.10)
    assert (r["sm_mhz"], r["samples"], r["reasons"]) == (1932.5, 2, ["hw_slowdown"])
    assert r["window"] == "timed region +- 0.25 s"
