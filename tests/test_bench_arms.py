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
