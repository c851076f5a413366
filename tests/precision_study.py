"""Precision study (checker side): error of every update variant against FP64
across a conditioning sweep.

Workload: the single-seed endcap track and hit of the pseudocode
(tests/golden/readme_seed.txt), every element smeared by (1 + 1e-5 N(0,1)),
20 layers.  Conditioning is swept by scaling the track's q/pT uncertainty
(sigma(q/pT)/|q/pT| from 1e-1 to 1e-6, its covariance row and column rescaled
so that correlations are kept) and the hit's transverse uncertainty (sigma
from 1 cm to 1 um, the xy block of V rescaled, its x-y correlation of -0.9988
kept).  The hit's x-z and y-z covariances are set to zero: with the seed's own
values (correlations of about 0.03 against sigma_z = 3.4 cm) the 3x3 hit
covariance is near-singular once its xy block is rescaled (condition number
1.2e7 at 1 cm to 1.2e13 at 10 um), which only the 3-D update reads and which
makes that problem ill-posed in any precision; the 2-D updates never read
them.  For each point the table gives, at the first update of track 0, the
condition number of R = C + V (xy block, C propagated) and the ratio of the
track's to the hit's xy sigma, which sets how much the update shrinks C and so
how much cancellation C - K H C suffers.

References:
  * 2-D variants: the GPU FP64 kernel on all tracks (itself pinned to the FP64
    host oracle, agreement printed per point);
  * 3-D (3x3 + Joseph) variants: the FP64 host oracle's 3x3 Joseph update on
    the first `--oracle-tracks` tracks;
  * "float-state floor": the FP64 host oracle run one layer at a time with the
    track state rounded to FP32 between layers -- the error any variant that
    stores its state in FP32 (every variant but full FP64) starts from.
Metrics as in the tests: parameters |d|/max(|ref|, floor), covariance
|dC_ij|/sqrt(C_ii C_jj).

    python tests/precision_study.py --tracks 2000000 --out profiles/precision_study.md
"""
from __future__ import annotations

import argparse
import pathlib
import sys
import time

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parent / "oracle"))

import conftest  # noqa: E402
import oracle as O  # noqa: E402

SIG_IPT = [1e-1, 1e-2, 1e-3, 1e-4, 1e-5, 1e-6]
SIG_HIT_CM = [1.0, 1e-1, 1e-2, 1e-3, 1e-4]
VARIANTS = [("reference FP32", "v2", 0x20), ("precise FP32", "v2", 0), ("FP64-free compensated", "v2_comp", 0),
            ("3x3 FP64 island + Joseph", "3x3_f64", 0), ("3x3 compensated FP32", "3x3_comp", 0),
            ("full FP64", "f64", 0)]
COLUMNS = [v[0] for v in VARIANTS] + ["float-state floor (2d)", "float-state floor (3x3)"]


def base_workload(p2z, ntracks):
    """Smeared README-seed tracks and hits at the seed's own uncertainties."""
    trk0, hits0 = conftest.read_seed(HERE / "golden" / "readme_seed.txt")
    par, cov, q = trk0
    hits = [hits0[0]] * 20
    ntr = (ntracks // 32) * 32
    trk, hit = p2z.prepare(p2z.make_atrk(par, cov, q), p2z.make_ahits(hits), 32, 1, ntr, 20, smear=1e-5,
                           cov_scale=1.0)
    return trk, hit, par, cov, hits0[0][1]


IPT_ROW = [6, 7, 8, 13, 18]  # packed (3,0) (3,1) (3,2) (4,3) (5,3)
IPT_DIAG = 9


def conditioned(trk, hit, par, cov, hcov, sig_ipt, sig_hit):
    """Rescale the smeared arrays (the smear is multiplicative, so this equals
    smearing rescaled seeds): the q/pT row and column of every track covariance
    by f, its diagonal by f^2, with sigma(q/pT) = sig_ipt |q/pT| at the seed;
    the hit xy block by g, xz and yz by sqrt(g), with sigma_xy = sig_hit."""
    f = sig_ipt * abs(par[3]) / np.sqrt(cov[IPT_DIAG])
    g = sig_hit ** 2 / np.sqrt(hcov[0] * hcov[2])
    t = trk.copy()
    t[:, [6 + k for k in IPT_ROW], :] *= np.float32(f)
    t[:, 6 + IPT_DIAG, :] *= np.float32(f * f)
    h = hit.copy()
    h[:, :, 3:6, :] *= np.float32(g)
    h[:, :, 6:8, :] = 0.0  # x-z and y-z hit covariances (see the module text)
    # the first update's inputs, for track 0: propagated C (xy block) and V
    b = np.ascontiguousarray(t[0])
    O.step_f32(b, np.ascontiguousarray(h[0, 0]), 0)
    Cxy = np.array([[b[6, 0], b[7, 0]], [b[7, 0], b[8, 0]]], dtype=np.float64)
    V = np.array([[h[0, 0, 3, 0], h[0, 0, 4, 0]], [h[0, 0, 4, 0], h[0, 0, 5, 0]]], dtype=np.float64)
    cond = float(np.linalg.cond(Cxy + V))
    shrink = float(np.sqrt(np.trace(Cxy) / np.trace(V)))  # track sigma / hit sigma in xy
    return t, h, cond, shrink


def _aos(torch, d):
    nb, w, B = d.shape
    a = d.permute(0, 2, 1).reshape(nb * B, w)
    return a[:, :6].double(), a[:, 6:27].double()


def errors_gpu(torch, out, ref_par, ref_cov):
    """The tests' metrics, evaluated on the device over every track."""
    par, cov = _aos(torch, out)
    floor = torch.tensor(conftest.PAR_FLOOR, dtype=torch.float64, device=out.device)
    finite = torch.isfinite(par).all(1) & torch.isfinite(ref_par).all(1)
    pr = ((par - ref_par).abs() / torch.maximum(ref_par.abs(), floor))[finite]
    diag = [i * (i + 1) // 2 + i for i in range(6)]
    cr = []
    for k in conftest.LIVE:
        i = int((np.sqrt(8 * k + 1) - 1) // 2)
        j = k - i * (i + 1) // 2
        s = (ref_cov[:, diag[i]] * ref_cov[:, diag[j]]).abs().sqrt()
        cr.append(((cov[:, k] - ref_cov[:, k]).abs() / torch.where(s > 0, s, torch.ones_like(s)))[finite])
    cr = torch.stack(cr, 1)
    q99 = lambda x: float(x.flatten().sort().values[max(0, int(0.99 * x.numel()) - 1)])
    return {"par_max": pr.max(0).values.cpu().numpy(), "cov_max": float(cr.max()), "cov_p99": q99(cr),
            "nonfinite": int((~torch.isfinite(par).all(1)).sum())}


def float_state_floor(p2z, trk, hit, update):
    """FP64 oracle, one layer at a time, state rounded to FP32 in between."""
    nb, w, B = trk.shape
    cur = trk.copy()
    for l in range(hit.shape[1]):
        o = O.run_f64(cur, np.ascontiguousarray(hit[:, l:l + 1]), update=update)
        cur[:, :27, :] = o.reshape(nb, B, 27).astype(np.float32).transpose(0, 2, 1)
    return cur


def errors_host(p2z, out, ref64):
    g = p2z.tracks_to_aos(out)
    finite = np.isfinite(g["par"]).all(1) & np.isfinite(ref64[:, :6]).all(1)
    pr = conftest.par_rel(g["par"][finite], ref64[finite, :6])
    cr = conftest.cov_rel(g["cov"][finite], ref64[finite, 6:])[:, conftest.LIVE]
    return {"par_max": pr.max(0), "cov_max": float(cr.max()), "cov_p99": float(np.percentile(cr, 99)),
            "nonfinite": int((~np.isfinite(g["par"]).all(1)).sum())}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--tracks", type=int, default=2_000_000)
    ap.add_argument("--oracle-tracks", type=int, default=8192)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    p2z = conftest.load_p2z()
    import torch
    ctx = p2z.Context(0)
    rows = []
    t0 = time.time()
    base_t, base_h, par, cov, hcov = base_workload(p2z, args.tracks)
    B = 32
    ntr = base_t.shape[0] * B
    nb_o = args.oracle_tracks // B
    cfg = lambda upd, fl: p2z.make_config(bsize=B, nevts=1, ntrks=ntr, nlayer=20, update=upd, flags=fl)
    for si in SIG_IPT:
        for sh in SIG_HIT_CM:
            trk, hit, cond, shrink = conditioned(base_t, base_h, par, cov, hcov, si, sh)
            dt, dh = torch.from_numpy(trk).cuda(), torch.from_numpy(hit).cuda()
            do = torch.empty_like(dt)
            ctx.run_device(cfg("f64", 0), dt, dh, do)
            torch.cuda.synchronize()
            ref_par, ref_cov = _aos(torch, do)
            f64_host = do[:nb_o].cpu().numpy()
            to, ho = np.ascontiguousarray(trk[:nb_o]), np.ascontiguousarray(hit[:nb_o])
            o2 = O.run_f64(to, ho)
            o3 = O.run_f64(to, ho, update=O.UPDATE_3X3_JOSEPH)
            f64_vs_oracle = errors_host(p2z, f64_host, o2)
            floors = {"2d": errors_host(p2z, float_state_floor(p2z, to, ho, O.UPDATE_V2), o2),
                      "3x3": errors_host(p2z, float_state_floor(p2z, to, ho, O.UPDATE_3X3_JOSEPH), o3)}
            for kind, e in floors.items():
                rows.append({"sig_ipt": si, "sig_hit_cm": sh, "cond": cond, "shrink": shrink,
                             "variant": f"float-state floor ({kind})", **e, "f64_vs_oracle_par_max": 0.0})
            for name, upd, fl in VARIANTS:
                out = torch.empty_like(dt)
                ctx.run_device(cfg(upd, fl), dt, dh, out)
                torch.cuda.synchronize()
                if upd.startswith("3x3"):
                    e = errors_host(p2z, out[:nb_o].cpu().numpy(), o3)
                else:
                    e = errors_gpu(torch, out, ref_par, ref_cov)
                rows.append({"sig_ipt": si, "sig_hit_cm": sh, "cond": cond, "shrink": shrink, "variant": name, **e,
                             "f64_vs_oracle_par_max": float(f64_vs_oracle["par_max"].max())})
                del out
            print(f"sig_ipt {si:g} sig_hit {sh:g} cm cond {cond:.1e} shrink {shrink:.1e} done ({time.time() - t0:.0f} s)", flush=True)
            del dt, dh, do, ref_par, ref_cov
    ctx.close()
    names = ["x", "y", "z", "ipt", "phi", "theta"]
    lines = ["# Precision study: every update variant against FP64 across a conditioning sweep", "",
             "Generated by `python tests/precision_study.py --tracks %d --out <this file>` on one B200." % args.tracks,
             "", __doc__.split("\n\n")[1], "", __doc__.split("\n\n")[2], "",
             "Rows: sigma(q/pT) relative; hit sigma (cm); at the first update of track 0, the condition number of R = C + V "
             "(xy block, C propagated) and the ratio sigma_track/sigma_hit in xy (how far the update shrinks C).",
             f"2-D variants against the GPU FP64 kernel on all {ntr} tracks; 3x3 variants against the "
             f"FP64 host oracle's 3x3 Joseph update on the first {nb_o * B} tracks; float-state floors on "
             f"those {nb_o * B} tracks.",
             "Cells: max relative error of the worst parameter / max normalised covariance error "
             "(non-finite tracks in brackets when any).", ""]
    hdr = "| sigma(q/pT) | hit sigma | cond(R) | track/hit sigma | " + " | ".join(COLUMNS) + " |"
    lines += [hdr, "|" + "---|" * (4 + len(COLUMNS))]
    for si in SIG_IPT:
        for sh in SIG_HIT_CM:
            rs = [r for r in rows if r["sig_ipt"] == si and r["sig_hit_cm"] == sh]
            cells = []
            for name in COLUMNS:
                r = next(x for x in rs if x["variant"] == name)
                c = f"{r['par_max'].max():.1e} / {r['cov_max']:.1e}"
                if r["nonfinite"]:
                    c += f" [{r['nonfinite']}]"
                cells.append(c)
            lines.append(f"| {si:g} | {sh:g} | {rs[0]['cond']:.1e} | {rs[0]['shrink']:.1e} | " + " | ".join(cells) + " |")
    lines += ["", "Per-parameter maxima (x, y, z, ipt, phi, theta) at every point:", ""]
    lines += ["| sigma(q/pT) | hit sigma | variant | " + " | ".join(names) + " | cov p99 |",
              "|---|---|---|" + "---|" * 7]
    for r in rows:
        lines.append(f"| {r['sig_ipt']:g} | {r['sig_hit_cm']:g} | {r['variant']} | " +
                     " | ".join(f"{v:.1e}" for v in r["par_max"]) + f" | {r['cov_p99']:.1e} |")
    lines += ["", "GPU FP64 kernel vs FP64 host oracle, 2-D update (worst parameter, per point): " +
              ", ".join(f"{r['f64_vs_oracle_par_max']:.1e}" for r in rows if r["variant"] == "full FP64")]
    text = "\n".join(lines) + "\n"
    if args.out:
        pathlib.Path(args.out).write_text(text)
    print(text)


if __name__ == "__main__":
    main()
