"""Regenerates the golden fixtures in this directory from the reference itself.

Run in a container that has the reference tree (default /root/reference) and
the reference built by ``make -C oracle ref``:

    python tests/golden/make_golden.py [REFERENCE_ROOT]

Outputs (all small, committed):
  kat_seed.txt        the reference's known-answer seed (src/input_track.h),
                      read through the reference's compiled code
                      (ref_kat_seed), one line for the track and one per hit
                      in the layer order of the reference's main (:693-695).
  readme_seed.txt     the single-seed workload's track and hit, parsed from
                      propagate-toz-pseudocode.txt:1-19, the hit repeated on
                      20 layers.
  kat_block.json      the validation block of the reference's golden log
                      logs/propagate_gcc_omp.log:30-40 (and the TBB and
                      icc-strict logs), with the run sizes.
  ref_kat_small.npz   per-track outputs of the reference's hot loop on its
                      2 x 128-track prepared KAT input, built with FMA
                      contraction (its Makefile flags) and without.
  ref_readme_small.npz  the same for the single-seed workload (smear 1e-5,
                      covariance scale 1).
"""
from __future__ import annotations

import json
import pathlib
import re
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "oracle"))
import oracle as O  # noqa: E402

REF = pathlib.Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")


def write_seed(path, trk, hits):
    with open(path, "w") as f:
        f.write(" ".join(repr(float(v)) for v in trk[0]) + " " + " ".join(repr(float(v)) for v in trk[1]) +
                f" {int(trk[2])}\n")
        for pos, cov in hits:
            f.write(" ".join(repr(float(v)) for v in list(pos) + list(cov)) + "\n")


def read_seed(path):
    lines = [l.split() for l in open(path) if l.strip()]
    t = lines[0]
    trk = ([float(v) for v in t[:6]], [float(v) for v in t[6:27]], int(t[27]))
    hits = [([float(v) for v in l[:3]], [float(v) for v in l[3:9]]) for l in lines[1:]]
    return trk, hits


def parse_block(text):
    out = {}
    for key, pat in [("x", r"track x avg=(\S+) std/avg=(\S+)"), ("y", r"track y avg=(\S+) std/avg=(\S+)"),
                     ("z", r"track z avg=(\S+) std/avg=(\S+)"), ("dx", r"track dx/x avg=(\S+) std=(\S+)"),
                     ("dy", r"track dy/y avg=(\S+) std=(\S+)"), ("dz", r"track dz/z avg=(\S+) std=(\S+)")]:
        m = re.search(pat, text)
        out[key] = [m.group(1), m.group(2)]
    for key, pat in [("pt", r"track pt avg=(\S+)"), ("phi", r"track phi avg=(\S+)"),
                     ("theta", r"track theta avg=(\S+)"), ("nans", r"number of tracks with nans=(\S+)"),
                     ("failed", r"number of tracks failed=(\S+)")]:
        out[key] = re.search(pat, text).group(1)
    return out


def main():
    # 1. KAT seed through the reference's compiled code
    trk, hits = O.ref_kat_seed()
    write_seed(HERE / "kat_seed.txt", trk, hits)

    # 2. the pseudocode seed: numbers after "par =" / "cov =" / "q =" of the
    #    input track, then of the input hit
    text = (REF / "propagate-toz-pseudocode.txt").read_text()
    blocks = re.findall(r"par\s*=\s*\{([^}]*)\}", text)
    covs = re.findall(r"cov\s*=\s*\{([^}]*)\}", text)
    q = int(re.search(r"q\s*=\s*(-?\d+)", text).group(1))
    tpar = [float(v) for v in blocks[0].split(",")]
    tcov = [float(v) for v in covs[0].split(",")]
    hpos = [float(v) for v in blocks[1].split(",")]
    hcov = [float(v) for v in covs[1].split(",")]
    assert len(tpar) == 6 and len(tcov) == 21 and len(hpos) == 3 and len(hcov) == 6
    write_seed(HERE / "readme_seed.txt", (tpar, tcov, q), [(hpos, hcov)] * 20)

    # 3. golden validation blocks
    logs = {}
    for name in ("propagate_gcc_omp.log", "propagate_gcc_tbb.log", "propagate_icc-strict_tbb.log"):
        logs[name] = parse_block((REF / "logs" / name).read_text())
    meta = {"nevts": 100, "ntrks": 9600, "bsize": 32, "nlayer": 20, "smear": 1e-7, "cov_scale": 100.0,
            "source": "logs/propagate_gcc_omp.log:30-40", "blocks": logs}
    (HERE / "kat_block.json").write_text(json.dumps(meta, indent=1) + "\n")

    # 4. per-track reference outputs on the small prepared KAT input
    trk_seed, hit_seeds = read_seed(HERE / "kat_seed.txt")
    t, h = O.ref_prepare("b32", trk_seed, hit_seeds)
    out_fma = O.ref_run(t, h, name="b32")
    out_nofma = O.ref_run(t, h, name="b32_nofma")
    np.savez_compressed(HERE / "ref_kat_small.npz", out_fma=out_fma, out_nofma=out_nofma,
                        note="reference hot loop on srand(1) prepareTracks/prepareHits, 2 events x 128 tracks, "
                             "bsize 32, 20 layers, smear 1e-7, cov x100")

    # 5. single-seed workload, smear 1e-5, covariance unscaled: inputs come from
    #    the library's reference-compatible generator (bit-exact with the
    #    reference's prepare, checked by the tests), outputs from the reference.
    import importlib.util
    spec = importlib.util.spec_from_file_location("p2z_b200", ROOT / "p2z-tests_b200" / "__init__.py",
                                                  submodule_search_locations=[str(ROOT / "p2z-tests_b200")])
    p2z = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(p2z)
    rs, rh = read_seed(HERE / "readme_seed.txt")
    t, h = p2z.prepare(p2z.make_atrk(*rs), p2z.make_ahits(rh), 32, 2, 128, 20, smear=1e-5, cov_scale=1.0)
    np.savez_compressed(HERE / "ref_readme_small.npz", out_fma=O.ref_run(t, h, name="b32"),
                        out_nofma=O.ref_run(t, h, name="b32_nofma"),
                        note="reference hot loop on the pseudocode seed, 2 x 128 tracks, smear 1e-5, cov x1")
    # 6. the validation block of the FP64 host oracle on the full known-answer
    #    input (100 x 9600): what an exact evaluation of the reference's
    #    algorithm prints; the golden log's FP32 evaluation differs from it in
    #    the 5th-6th significant digit.
    t, h = p2z.prepare(p2z.make_atrk(*trk_seed), p2z.make_ahits(hit_seeds), 32, 100, 9600, 20)
    o64 = O.run_f64(t, h)
    a = t.copy()
    a[:, :27, :] = o64.reshape(t.shape[0], 32, 27).transpose(0, 2, 1).astype(np.float32)
    v = p2z.validate(a, 32, 100, 9600, hit_seeds[19][0])
    meta["fp64_block"] = {k: "%f" % getattr(v, k) for k in ("avgx", "avgy", "avgz", "avgdx", "avgdy", "avgpt",
                                                            "avgphi", "avgtheta")}
    meta["fp64_block"]["source"] = "FP64 host oracle (oracle/p2z_oracle.c) on the 100 x 9600 known-answer input"
    (HERE / "kat_block.json").write_text(json.dumps(meta, indent=1) + "\n")
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
