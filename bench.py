"""Benchmark: track-layer updates/s of the propagate-to-z + Kalman-update hot
path on B200 (one JSON line on rank 0).

Workload (one GPU): 1000 events x 9600 tracks, 20 layers, FP32, bsize-32
AOSOA -- the physics workload (charge +-1, pT log-uniform 0.5-20 GeV, phi
uniform, eta 1.6-2.5, vertex z ~ N(0, 5 cm), correlated PD covariances, hits on
20 planes z = 30..270 cm at the true helix point plus 30 um / 1 um noise),
generated from a fixed seed on the device (p2z_generate_physics_device).  A step is one pass of the hot path over all 9.6M
tracks x 20 layers.  Inputs (8.1 GB) are larger than L2, so no flush is needed.

  value   device-resident throughput (p2z_run_device, CUDA events on the stream)
  e2e     the same metric through p2z_run from pinned host buffers, host->device
          and device->host copies inside the timed region
  batched_vs_plain  uneven events (2000 events, log-normal track counts,
          5-20 hits per track with 10% of layers dropped): the persistent
          work-queue kernel replayed as a CUDA graph vs one launch per event,
          each with the block size the autotuner measured best for it
  autotune  p2z_autotune's sweep (bsize x AOSOA/SoA x schedule x block size x
          threads per track) on the headline and the uneven workloads; the
          headline step runs the reference's layout (bsize 32 AOSOA) with the
          schedule, block size and threads per track the sweep found best for
          that layout
  threads_per_track  one against two threads per track: headline
          throughput, and the device time of one launch over a lone event of
          1024, 3072 or 9600 tracks

`--impl reference` times the reference's own CPU hot loop (its OpenMP source
compiled unchanged into oracle/_ref) on this host's cores, on the same
workload, one bounded sample of events per step.

Multi-GPU (torchrun): every rank runs its own 1000 events (weak scaling, no
data-path collective); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import pathlib
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent

# Algorithmic work per track-layer update (reduced form, z row zero):
#   FP32 flops (FMA = 2): propagation scalars 30 + Jacobian 55 + J C J^T 142
#   + 2-D Kalman update 122 = 349.
#   Compulsory bytes: 6 hit words (24 B) + track in and out (2 x 112 B) over
#   20 layers (11.2 B) = 35.2 B.
FLOPS_PER_UPDATE = 349
# The same update counted as the reference writes it (its propagateToZ
# scalars, the full MultHelixPropEndcap / MultHelixPropTranspEndcap products
# including those with J's known zeros, KalmanUpdate_v2): ~460 FP32 flops.
# Reported beside the reduced count, never in place of it.
FLOPS_PER_UPDATE_REFERENCE_FORM = 460
BYTES_PER_UPDATE = 35.2
BYTES_HIT_PER_UPDATE = 24   # the 6 hit words a 2-D update reads
BYTES_TRACK = 228           # a track read and written (2 x 112 B) and its mask word
FP32_LANES_PER_SM = 128

METRIC = "track-layer updates/s on 1 B200, batched vs plain, <=1e-5 rel err vs FP64"
WORKLOAD = "physics 1000 events x 9600 tracks x 20 layers, bsize 32, FP32"


def load_p2z():
    pkg = ROOT / "p2z-tests_b200"
    spec = importlib.util.spec_from_file_location("p2z_b200", pkg / "__init__.py",
                                                  submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["p2z_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d.get("hbm_gbs"), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def profile_traffic_per_update():
    """dram bytes per update from the committed ncu summary of the kernel, if any."""
    p = ROOT / "profiles" / "k_flat_v2_physics.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("dram_bytes_per_update:"):
            return float(line.split(":")[1])
    return None


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed
    region: NVML polled every 2 ms from a thread (the data nvidia-smi reports),
    or nvidia-smi -lms 200 when NVML is unavailable."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40, "sw_power_cap": 0x4}

    def __init__(self, cuda_index):
        self.cuda_index = cuda_index
        self.samples = []       # (time, sm_mhz, reasons bitmask)
        self.sm_max = None
        self.power_w = []
        self._stop = threading.Event()
        self._thread = None
        self._nvml = None
        self._handle = None
        self._proc = None
        self._lines = []

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        self._nvml = pynvml
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.cuda_index).uuid)
            return pynvml.nvmlDeviceGetHandleByUUID(("GPU-" + uuid) if not uuid.startswith("GPU-") else uuid)
        except Exception:
            pass
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        idx = self.cuda_index
        if vis:
            try:
                idx = int(vis.split(",")[self.cuda_index])
            except (ValueError, IndexError):
                pass
        return pynvml.nvmlDeviceGetHandleByIndex(idx)

    def start(self):
        try:
            self._handle = self._nvml_handle()
            nv = self._nvml
            self.sm_max = float(nv.nvmlDeviceGetMaxClockInfo(self._handle, nv.NVML_CLOCK_SM))
            self._thread = threading.Thread(target=self._poll, daemon=True)
            self._thread.start()
            # return once the thread is sampling, so that the timed region that follows is covered
            t_end = time.perf_counter() + 1.0
            while len(self.samples) < 3 and self._thread.is_alive() and time.perf_counter() < t_end:
                time.sleep(0.001)
            return
        except Exception:
            self._nvml = None
        try:
            fields = "clocks.sm,clocks.max.sm,clocks_event_reasons.active"
            self._proc = subprocess.Popen(["nvidia-smi", f"--id={self.cuda_index}", f"--query-gpu={fields}",
                                           "--format=csv,noheader,nounits", "-lms", "200"],
                                          stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=lambda: self._lines.extend(l.strip() for l in self._proc.stdout),
                             daemon=True).start()
        except OSError:
            self._proc = None

    def _poll(self):
        nv, h = self._nvml, self._handle
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self._stop.is_set():
            try:
                self.samples.append((time.perf_counter(), float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                     int(get_reasons(h))))
                if len(self.samples) % 25 == 1:
                    self.power_w.append(nv.nvmlDeviceGetPowerUsage(h) / 1000.0)
            except Exception:
                break
            time.sleep(0.002)

    def stop(self, t0=None, t1=None):
        """Summary of the samples taken between host times t0 and t1 (the
        timed region; all samples when not given)."""
        self._stop.set()
        if self._thread is not None:
            self._thread.join(timeout=2)
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()
            for l in self._lines:
                f = [x.strip() for x in l.split(",")]
                try:
                    self.sm_max = float(f[1])
                    self.samples.append((None, float(f[0]), int(f[2], 16)))
                except (ValueError, IndexError):
                    continue
        sel = [x for x in self.samples if x[0] is None or t0 is None or t0 <= x[0] <= t1]
        window = "timed region"
        if not sel and t0 is not None:
            # a timed region shorter than the sampler's period: the samples nearest to it
            sel = [x for x in self.samples if x[0] is not None and t0 - 0.25 <= x[0] <= t1 + 0.25]
            window = "timed region +- 0.25 s"
        sm = [a for _, a, _ in sel]
        mask = 0
        for _, _, r in sel:
            mask |= r
        reasons = sorted(n for n, bit in self.REASONS.items() if mask & bit)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": self.sm_max, "reasons": reasons,
                "samples": len(sm), "window": window, "source": "nvml" if self._nvml else "nvidia-smi",
                "power_w_median": float(np.median(self.power_w)) if self.power_w else None}


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        import torch
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier_max(world, value):
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def order_by_hits(torch, counts, udt, udh, udm):
    """Copies of an uneven sample with each event's tracks in order of their hit
    count (most hits first, padding slots last) and the slot permutation.  A
    32-track batch runs as one warp, which takes as many steps as its longest
    track, so batches of similar-length tracks keep every lane busy; callers
    get this by ordering tracks when they pack an event's batches."""
    nslots = udm.numel()
    nb, nlayer = udh.shape[0], udh.shape[1]
    m = udm.to(torch.int64) & 0xFFFFFFFF
    pc = torch.zeros(nslots, dtype=torch.int64, device=udm.device)
    for b in range(32):
        pc += (m >> b) & 1
    per_event = torch.as_tensor(((counts + 31) // 32) * 32, device=udm.device)
    ev = torch.repeat_interleave(torch.arange(len(counts), device=udm.device), per_event)
    perm = torch.sort(ev * 64 + (32 - pc), stable=True).indices
    ts = udt.permute(0, 2, 1).reshape(nslots, -1)[perm].reshape(nb, 32, -1).permute(0, 2, 1).contiguous()
    hs = udh.permute(0, 3, 1, 2).reshape(nslots, nlayer, -1)[perm]
    hs = hs.reshape(nb, 32, nlayer, -1).permute(0, 2, 3, 1).contiguous()
    util = lambda x: float(x.sum()) / float(32 * x.reshape(-1, 32).max(1).values.sum())
    return ts, hs, udm[perm].contiguous(), perm, util(pc), util(pc[perm])


def window_util(mask, win):
    """Lane utilisation of a masked run whose `win`-slot windows are processed
    in order of hit count: present-hit lane-steps over 32 x the warps' steps."""
    import torch
    m = mask.to(torch.int64) & 0xFFFFFFFF
    pc = torch.zeros_like(m)
    for b in range(32):
        pc += (m >> b) & 1
    n = (pc.numel() + win - 1) // win * win
    pc = torch.nn.functional.pad(pc, (0, n - pc.numel()))
    s = torch.sort(pc.view(-1, win), dim=1, descending=True).values
    return float(pc.sum()) / float(32 * s.view(-1, 32).max(1).values.sum())


def uneven_counts(n_events, seed):
    rng = np.random.default_rng(seed)
    c = np.exp(np.log(3000.0) + 1.0 * rng.standard_normal(n_events))
    return np.clip(np.rint(c), 50, 30000).astype(np.int64)


# ---------------------------------------------------------------------------
# serving
# ---------------------------------------------------------------------------

SERVE_RATES = (1000, 2000, 5000, 10000, 20000, 50000)


def tune_summary(best, rows, wall_s):
    """Compact report of an autotune sweep: the fastest row overall, per bsize,
    per layout and per schedule, and the row the reference's layout gets."""
    def fastest(pred):
        sel = [r for r in rows if pred(r)]
        return min(sel, key=lambda r: r["ms"]) if sel else None
    out = {"configurations": len(rows), "sweep_wall_s": wall_s, "best": best,
           "best_bsize32_aosoa": fastest(lambda r: r["bsize"] == 32 and r["layout"] == "aosoa")}
    for key in ("bsize", "layout", "schedule", "threads_per_track", "sorted_windows"):
        vals = sorted({r[key] for r in rows}, key=str)
        out[f"best_per_{key}"] = {str(v): {"ms": fastest(lambda r: r[key] == v)["ms"],
                                           "updates_per_s": fastest(lambda r: r[key] == v)["updates_per_s"]}
                                  for v in vals}
    return out


def small_run_latency(p2z, ctx, t, h, o):
    """Host wall time of one synchronous p2z_run call on a lone event of 1024
    or 9600 tracks from page-locked buffers (the first batches of the bench
    sample): the default call -- a pipeline of 4 or more chunk passes (9600
    tracks: 4 chunks) replayed as a recorded graph, a shorter one (1024
    tracks: 1 chunk) enqueued directly -- against the same pipeline always
    enqueued copy by copy (P2Z_FLAG_NO_GRAPH); mean of 200 calls after 5
    warm-up calls."""
    out = {}
    for n in (1024, 9600):
        nb = n // 32
        row = {}
        for mode, flags in (("default", 0), ("direct", p2z.FLAG_NO_GRAPH)):
            cfg = p2z.make_config(bsize=32, nevts=1, ntrks=n, nlayer=20, schedule="flat", flags=flags)
            args = (ctx.h, p2z.C.byref(cfg), t[:nb].ctypes.data, h[:nb].ctypes.data, None, o[:nb].ctypes.data, None)
            for _ in range(5):
                p2z.lib.p2z_run(*args)
            t0 = time.perf_counter()
            for _ in range(200):
                rc = p2z.lib.p2z_run(*args)
            us = (time.perf_counter() - t0) / 200 * 1e6
            if rc != p2z.OK:
                raise p2z.P2zError(rc, p2z.lib.p2z_last_error(ctx.h).decode())
            row[mode + "_us"] = us
        out[str(n)] = row
    return {"note": "p2z_run from page-locked buffers, one event, host wall time per synchronous call; default: "
                    "recorded graph from 4 chunk passes (9600 tracks), direct below (1024 tracks)",
            "tracks": out}


def threads_per_track_report(p2z, ctx, torch, dt, dh, do, stream):
    """One thread per track against two (p2z_config.threads_per_track), flat
    launches of the precise form at bsize 32 AOSOA: (1) throughput on the
    headline sample, best block size each; (2) the device time of one launch
    over a lone event of 1024, 3072 or 9600 tracks (the first batches of the
    sample), where the GPU is mostly empty and a track's 20-layer chain sets
    the time.  The lone-event time is the mean over 200 launches queued back
    to back on one stream behind a sleep kernel (so that host submission does
    not enter the timed span), between one pair of CUDA events: the kernel's
    duration plus the gap between consecutive kernels.  (Events around each
    launch would read in steps of the timer's 2.048 us resolution.)"""
    def launcher(cfg, t, h, o):
        args = (ctx.h, p2z.C.byref(cfg), t.data_ptr(), h.data_ptr(), None, o.data_ptr(),
                p2z.C.c_void_p(stream.cuda_stream), None)
        def go():
            rc = p2z.lib.p2z_run_device(*args)
            if rc != p2z.OK:
                raise p2z.P2zError(rc, p2z.lib.p2z_last_error(ctx.h).decode())
        return go

    nev = dt.shape[0] * 32 // 9600
    head = {}
    for tpt in (1, 2):
        best = None
        for block in (32, 64, 128, 256):
            cfg = p2z.make_config(bsize=32, nevts=nev, ntrks=9600, nlayer=20, schedule="flat", block_threads=block,
                                  threads_per_track=tpt)
            go = launcher(cfg, dt, dh, do)
            for _ in range(2):
                go()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(5):
                go()
            b.record(stream)
            torch.cuda.synchronize()
            ms = a.elapsed_time(b) / 5
            if best is None or ms < best["ms"]:
                best = {"ms": ms, "block_threads": block, "updates_per_s": nev * 9600 * 20 / (ms / 1e3)}
        head[str(tpt)] = best
    lone = {}
    for n in (1024, 3072, 9600):
        nb = n // 32
        row = {}
        for tpt in (1, 2):
            best = None
            for block in (32, 64, 128):
                cfg = p2z.make_config(bsize=32, nevts=1, ntrks=n, nlayer=20, schedule="flat", block_threads=block,
                                      threads_per_track=tpt)
                go = launcher(cfg, dt[:nb], dh[:nb], do[:nb])
                for _ in range(3):
                    go()
                reps = 200
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                with torch.cuda.stream(stream):
                    torch.cuda._sleep(40_000_000)  # ~20 ms: the queue fills while the GPU waits
                a.record(stream)
                for _ in range(reps):
                    go()
                b.record(stream)
                torch.cuda.synchronize()
                us = a.elapsed_time(b) * 1e3 / reps
                if best is None or us < best["us"]:
                    best = {"us": us, "block_threads": block}
            row[str(tpt)] = best
        row["ratio_1_over_2"] = row["1"]["us"] / row["2"]["us"]
        lone[str(n)] = row
    return {"note": "flat launches, precise form, bsize 32 AOSOA; two threads per track: lanes 2i and 2i+1 "
                    "hold the same track and split the propagation of its covariance (bit-identical results)",
            "headline": head, "headline_ratio_1_over_2": head["1"]["updates_per_s"] / head["2"]["updates_per_s"],
            "lone_event_launch_us": lone}


def run_serving(p2z, device, rank, args):
    """Events of 1k-20k tracks (log-uniform), 20 layers with missing-hit masks
    (5-20 hits, 10% dropped), the 3x3 update with its FP64 inversion island,
    admitted under a 40 GB ring; Poisson arrivals at each swept rate."""
    rng = np.random.default_rng(1234 + rank)
    npool = 128
    counts = np.exp(rng.uniform(np.log(1000), np.log(20000), npool)).astype(np.int64)
    pool = []
    for i, n in enumerate(counts):
        cfg = p2z.make_config(bsize=32, nevts=1, event_ntrks=[int(n)], nlayer=20)
        nb = p2z.num_batches(cfg)
        t = p2z.PinnedArray((nb, 28, 32))
        h = p2z.PinnedArray((nb, 20, 9, 32))
        m = p2z.PinnedArray((nb * 32,), np.uint32)
        o = p2z.PinnedArray((nb, 28, 32))
        p2z.generate_physics(cfg, p2z.physics_params(seed=5000 + i, nthreads=0), with_mask=True,
                             out=(t.array, h.array, m.array))
        p2z.mask_layers(m.array, 20, min_hits=5, max_hits=20, drop_prob=0.1, seed=77 + i)
        pool.append((t, h, m, o, int(n)))
    out = {"workload": "events of 1k-20k tracks (log-uniform), 20 layers, 5-20 hits/track with 10% dropped, "
                       "3x3 update with FP64 inversion + Joseph, Poisson arrivals",
           "device_budget_gb": 40, "events_per_rate": args.serve_events, "groups_in_flight": args.serve_inflight,
           "rates": []}
    with p2z.Server(device=device, bsize=32, nlayer=20, update="3x3_f64", budget_bytes=40 << 30,
                    max_inflight=args.serve_inflight) as srv:
        # warm-up
        srv.replay([(e[0].array, e[1].array, e[2].array, e[4], e[3].array) for e in pool[:16]],
                   np.zeros(16))
        rates = [int(r) for r in args.serve_rates.split(",")] if args.serve_rates else SERVE_RATES
        for rate in rates:
            n = args.serve_events
            idx = rng.integers(0, npool, n)
            arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
            evs = [(pool[i][0].array, pool[i][1].array, pool[i][2].array, pool[i][4], pool[i][3].array) for i in idx]
            infos = srv.replay(evs, arrivals)
            lat = np.array([x.done_s - x.submit_s for x in infos]) * 1e3
            span = max(x.done_s for x in infos) - min(x.submit_s for x in infos)
            upd = sum(x.updates for x in infos)
            out["rates"].append({
                "offered_events_per_s": rate, "events": n,
                "achieved_events_per_s": n / span, "updates_per_s": upd / span,
                "latency_ms_p50": float(np.percentile(lat, 50)), "latency_ms_p99": float(np.percentile(lat, 99)),
                "latency_ms_max": float(lat.max()),
                "mean_group_events": float(np.mean([x.group_events for x in infos]))})
    for e in pool:
        for a in e[:4]:
            a.free()
    return out


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------

def workload_config(nev, world):
    """The workload's description, identical in both arms."""
    gb = nev * 9600 * (28 + 20 * 9) * 4 / 1e9
    return {"workload": WORKLOAD if nev == 1000 else WORKLOAD.replace("1000 events", f"{nev} events"),
            "events": nev, "tracks_per_event": 9600, "nlayer": 20, "bsize": 32,
            "updates_per_step_per_gpu": nev * 9600 * 20,
            "l2": f"inputs {gb:.1f} GB {'>' if gb > 0.126 else '<'} L2, no flush",
            "parallelism": f"dp{world} (independent event shards)"}


def run_reference(args):
    """The reference's own OpenMP hot loop (src/propagate-toz-test_OMP.cpp
    compiled unchanged into oracle/_ref) on this host's cores.  Its inputs are
    the same physics sample, generated by the oracle's restatement of the
    generator: nothing of the product library is loaded in this arm."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    if not O.ref_available("b32"):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (needs the reference tree)"}))
        return 0
    cores = os.cpu_count() or 1
    n_ev = args.ref_events or cpu_sample_events(cores)
    trk, hit = O.physics(32, n_ev, 9600, 20, seed=20240601)
    upd = n_ev * 9600 * 20
    for _ in range(args.warmup):
        O.ref_run(trk, hit, nev=n_ev, nthreads=cores)
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.ref_run(trk, hit, nev=n_ev, nthreads=cores)
        ts.append(time.perf_counter() - t0)
    sec = float(np.sum(ts))
    value = upd * args.steps / sec
    sample = (f"{n_ev} of the {args.nevts} events x 9600 tracks x 20 layers per step "
              f"({upd} updates), OpenMP over events, {cores} threads")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args.nevts, world),
            "sample": {"events_per_step": n_ev, "updates_per_step": upd, "host_threads": cores,
                       "inputs": "the physics sample (seed 20240601) from the oracle's generator"},
            "cpu_baseline": {"value": value, "unit": "updates/s", "cores": cores, "kind": "reference",
                             "cpu_model": cpu_model(), "sample": sample},
            "e2e": {"value": value, "unit": "updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def reference_gpu(p2z, ctx, dt, dh, stream, launch):
    """The reference's own GPU build (src/propagate-toz-test_CUDA_v4.cu,
    unchanged, oracle/_ref/cuda_v4/p2z_cuda_v4_n100: 100 events x 9600 tracks
    x 20 layers, 200 passes, its kernels on 10 streams, device-resident data)
    run as its own process, and this library's kernel on the first 100 events
    of the bench sample, timed the reference's way: host wall clock around the
    200 passes and a final device synchronise."""
    import torch
    exe = ROOT / "oracle" / "_ref" / "cuda_v4" / "p2z_cuda_v4_n100"
    if not exe.exists():
        return None
    torch.cuda.synchronize()
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    fmt = [l.split() for l in r.stdout.splitlines() if l.startswith("formatted ")]
    if r.returncode != 0 or not fmt:
        return {"unavailable": f"exit {r.returncode}: {r.stderr[-200:]}"}
    niter, nev, ntrk, wall, setup = int(fmt[0][1]), int(fmt[0][2]), int(fmt[0][3]), float(fmt[0][6]), float(fmt[0][8])
    upd = nev * ntrk * 20
    cfg = p2z.make_config(bsize=32, nevts=nev, ntrks=ntrk, nlayer=20, schedule=launch["schedule"],
                          block_threads=launch["block_threads"])
    nb = nev * ntrk // 32
    t, h = dt[:nb], dh[:nb]
    o = torch.empty_like(t)
    args = (ctx.h, p2z.C.byref(cfg), t.data_ptr(), h.data_ptr(), None, o.data_ptr(),
            p2z.C.c_void_p(stream.cuda_stream), None)
    for _ in range(3):
        p2z.lib.p2z_run_device(*args)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(stream)
    for _ in range(niter):
        p2z.lib.p2z_run_device(*args)
    e1.record(stream)
    torch.cuda.synchronize()
    ours_wall = time.perf_counter() - t0
    ours_dev = e0.elapsed_time(e1) / 1e3
    return {"binary": "oracle/_ref/cuda_v4/p2z_cuda_v4_n100: src/propagate-toz-test_CUDA_v4.cu unchanged, its "
                      "Makefile's nvcc flags (MODE=cudav4, USE_ASYNC) for sm_100a, -Dnevts=100 -DNITER=200",
            "workload": f"{nev} events x {ntrk} tracks x 20 layers, {niter} passes, device-resident (its own "
                        "smeared known-answer input; this library: the first 100 events of the bench sample)",
            "reference_updates_per_s": upd * niter / wall, "reference_ms_per_pass": 1e3 * wall / niter,
            "reference_setup_s": setup,
            "ours_updates_per_s_wall": upd * niter / ours_wall, "ours_ms_per_pass_wall": 1e3 * ours_wall / niter,
            "ours_updates_per_s_device": upd * niter / ours_dev,
            "ratio_wall": wall / ours_wall}


def cpu_model():
    """The host CPU's model name (as lscpu reports it), or None."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_sample_events(cores):
    """Events in a CPU sample: a multiple of the thread count near 64, since
    the reference spreads whole events over its OpenMP threads (50 events on
    16 threads would leave the busiest thread 4 against an average of 3.1)."""
    return cores * max(1, round(64 / cores))


def cpu_baseline(p2z, trk, hit):
    """The reference's hot loop on this host's cores, on a bounded sample."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    if not O.ref_available("b32"):
        return None
    cores = os.cpu_count() or 1
    n_ev = cpu_sample_events(cores)
    nb = n_ev * 300
    t, h = np.ascontiguousarray(trk[:nb]), np.ascontiguousarray(hit[:nb])
    O.ref_run(t, h, nev=n_ev, nthreads=cores)
    reps, sec = 0, 0.0
    while sec < 10.0 and reps < 200:
        t0 = time.perf_counter()
        O.ref_run(t, h, nev=n_ev, nthreads=cores)
        sec += time.perf_counter() - t0
        reps += 1
    return {"value": n_ev * 9600 * 20 * reps / sec, "unit": "updates/s", "cores": cores, "kind": "reference",
            "cpu_model": cpu_model(),
            "sample": f"{n_ev} of the 1000 events, {reps} passes ({sec:.1f} s wall), reference OMP build, "
                      f"{cores} threads"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ref-events", type=int, default=0,
                    help="events per reference step (0: a multiple of the thread count near 64)")
    ap.add_argument("--nevts", type=int, default=1000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-uneven", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip running the reference's own CUDA_v4 build beside this kernel")
    ap.add_argument("--serve-events", type=int, default=1500)
    ap.add_argument("--serve-inflight", type=int, default=8, help="server groups in flight (1..8)")
    ap.add_argument("--serve-rates", default="", help="comma-separated offered rates (events/s); default sweep")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--no-lanes", action="store_true", help="skip the threads-per-track comparison")
    ap.add_argument("--schedule", default="auto", choices=["auto", "flat", "persistent", "per_event", "staged"],
                    help="launch schedule of the headline step (auto: what the autotuner measured best)")
    ap.add_argument("--block", type=int, default=0, help="threads per CTA of the headline step (0: tuned)")
    ap.add_argument("--threads-per-track", type=int, default=0, choices=[0, 1, 2],
                    help="threads per track of the headline step (0: tuned)")
    ap.add_argument("--update", default="v2", choices=["v2", "v2_comp", "3x3_f64", "3x3_comp", "f64"],
                    help="update kind of the headline step (v2: the precise 2-D form; the others for profiles)")
    ap.add_argument("--uneven-events", type=int, default=2000,
                    help="events of the uneven sample (2000: the config-4 workload; fewer for small profiles)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    import torch
    world, rank, local = dist_setup(args.gpus)
    torch.cuda.set_device(local)
    p2z = load_p2z()
    ctx = p2z.Context(local)
    # A stream of our own: its handle is never the legacy default stream (0),
    # which the C ABI would read as "the context's stream".
    stream = torch.cuda.Stream()
    # measured denominators on this GPU and its host link, before any timing
    live_peaks = p2z.measure_peaks(local)
    fp32_peak_live = max(live_peaks["fp32_ffma_tflops"], live_peaks["fp32_ffma2_tflops"])

    nev = args.nevts
    # schedule and block size left open: the context applies what p2z_autotune measured
    cfg = p2z.make_config(bsize=32, nevts=nev, ntrks=9600, nlayer=20, schedule=args.schedule,
                          block_threads=args.block, threads_per_track=args.threads_per_track, update=args.update)
    params = p2z.physics_params(seed=20240601 + rank)
    nb = p2z.num_batches(cfg)
    trk_shape, hit_shape = (nb, p2z.TRK_WORDS, 32), (nb, 20, p2z.HIT_WORDS, 32)
    # the physics sample generated where it is consumed (p2z_generate_physics_device:
    # the host generator's per-slot code on the GPU)
    dt = torch.empty(trk_shape, dtype=torch.float32, device="cuda")
    dh = torch.empty(hit_shape, dtype=torch.float32, device="cuda")
    ctx.generate_physics_device(cfg, dt, dh, params=params)
    updates = nev * 9600 * 20
    do = torch.empty_like(dt)
    # host copy of the first events for the CPU baseline (one GPU only: it measures the host's cores)
    n_cpu_ev = cpu_sample_events(os.cpu_count() or 1)
    cpu_sample = None
    if world == 1 and not args.no_cpu_baseline:
        cpu_sample = (dt[:n_cpu_ev * 300].cpu().numpy(), dh[:n_cpu_ev * 300].cpu().numpy())

    def step(c=cfg):
        rc = p2z.lib.p2z_run_device(ctx.h, p2z.C.byref(c), dt.data_ptr(), dh.data_ptr(), None, do.data_ptr(),
                                    p2z.C.c_void_p(stream.cuda_stream), None)
        if rc != p2z.OK:
            raise p2z.P2zError(rc, p2z.lib.p2z_last_error(ctx.h).decode())

    tune_head = None
    if not args.no_tune:
        t0 = time.time()
        best, rows = ctx.autotune(cfg, dt, dh, reps=3)
        tune_head = tune_summary(best, rows, time.time() - t0)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.05)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_begin = time.perf_counter()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    t_end = time.perf_counter()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop(t_begin, t_end)
    barrier(world)
    ms_max = barrier_max(world, ms)
    ms_step = ms_max / args.steps
    value = updates * world / (ms_step / 1e3)
    st = ctx.run_device(cfg, dt, dh, do)  # one more pass for the launch count and status
    launches_per_step = st.launches
    launch = {"schedule": (args.schedule if args.schedule != "auto" else
                           (tune_head["best_bsize32_aosoa"]["schedule"] if tune_head else "flat")),
              "block_threads": (args.block or (tune_head["best_bsize32_aosoa"]["block_threads"] if tune_head
                                               else 128)),
              "threads_per_track": (args.threads_per_track or
                                    (tune_head["best_bsize32_aosoa"]["threads_per_track"] if tune_head else 1))}
    ref_gpu = None
    if rank == 0 and not args.no_reference_gpu:
        ref_gpu = reference_gpu(p2z, ctx, dt, dh, stream, launch)
    lanes = None
    if rank == 0 and not args.no_lanes:
        lanes = threads_per_track_report(p2z, ctx, torch, dt, dh, do, stream)

    # e2e: host buffers through p2z_run
    e2e = None
    if not args.no_e2e:
        pin_t = p2z.PinnedArray(trk_shape)
        pin_h = p2z.PinnedArray(hit_shape)
        pin_o = p2z.PinnedArray(trk_shape)
        torch.from_numpy(pin_t.array).copy_(dt)
        torch.from_numpy(pin_h.array).copy_(dh)
        del dt, dh, do
        torch.cuda.empty_cache()
        ecfg = p2z.make_config(bsize=32, nevts=nev, ntrks=9600, nlayer=20, schedule="flat")
        for _ in range(3):
            ctx.run(ecfg, pin_t.array, pin_h.array, pin_o.array)
        barrier(world)
        tot = 0.0
        n_e2e = max(3, min(args.steps, 10))
        for _ in range(n_e2e):
            s = ctx.run(ecfg, pin_t.array, pin_h.array, pin_o.array)
            tot += s.total_ms
        tot = barrier_max(world, tot)
        e2e_ms = tot / n_e2e
        # the host link's floor for this step: each direction at its measured
        # pinned rate, and both together at the measured two-way rate
        link_ms = 1e3 * max(s.h2d_bytes / (live_peaks["h2d_gbs"] * 1e9), s.d2h_bytes / (live_peaks["d2h_gbs"] * 1e9),
                            (s.h2d_bytes + s.d2h_bytes) / (live_peaks["bidir_gbs"] * 1e9))
        e2e = {"value": updates * world / (e2e_ms / 1e3), "unit": "updates/s",
               "h2d_bytes_per_step": int(s.h2d_bytes), "d2h_bytes_per_step": int(s.d2h_bytes),
               "ms_per_step": e2e_ms, "steps": n_e2e,
               "path": "p2z_run, pinned host buffers, 16 chunks on 2 streams (copy/compute overlap)",
               "roofline": {"bound": "host link (PCIe)", "link_floor_ms": link_ms, "frac": link_ms / e2e_ms,
                            "ceiling_updates_per_s": updates * world / (link_ms / 1e3),
                            "peaks": {k: live_peaks[k] for k in ("h2d_gbs", "d2h_gbs", "bidir_gbs")},
                            "peak_source": "measured in this run: p2z_measure_peaks, one 1 GiB pinned "
                                           "cudaMemcpyAsync each way and both at once, best of 5"}}
        out_ok = bool(np.isfinite(pin_o.array[:, :6, :]).all())
        if rank == 0:
            e2e["small_runs"] = small_run_latency(p2z, ctx, pin_t.array, pin_h.array, pin_o.array)
        pin_t.free(); pin_h.free(); pin_o.free()
    else:
        del dt, dh, do
        out_ok = None
    torch.cuda.empty_cache()

    # batched (persistent + graph) vs plain (one launch per event) on uneven events
    bvp = None
    if not args.no_uneven:
        counts = uneven_counts(args.uneven_events, 77 + rank)
        ucfg = p2z.make_config(bsize=32, nevts=len(counts), event_ntrks=counts, nlayer=20)
        unb = p2z.num_batches(ucfg)
        udt = torch.empty((unb, p2z.TRK_WORDS, 32), dtype=torch.float32, device="cuda")
        udh = torch.empty((unb, 20, p2z.HIT_WORDS, 32), dtype=torch.float32, device="cuda")
        udm = torch.empty(unb * 32, dtype=torch.int32, device="cuda")
        ctx.generate_physics_device(ucfg, udt, udh, udm, params=p2z.physics_params(seed=99 + rank))
        ctx.mask_layers_device(udm, unb * 32, 20, min_hits=5, max_hits=20, drop_prob=0.1, seed=5 + rank)
        udo = torch.empty_like(udt)
        u_upd = int(ctx.run_device(ucfg, udt, udh, udo, d_mask=udm).updates)
        res, blocks = {}, {"persistent": 128, "per_event": 128}
        tune_uneven = None
        if not args.no_tune:
            t0 = time.time()
            best, rows = ctx.autotune(ucfg, udt, udh, d_mask=udm, reps=3)
            tune_uneven = tune_summary(best, rows, time.time() - t0)
            for sched in blocks:
                r = min((r for r in rows if r["bsize"] == 32 and r["layout"] == "aosoa" and r["schedule"] == sched),
                        key=lambda r: r["ms"])
                blocks[sched] = r["block_threads"]
        def timed(c, t, h, mk, o):
            """updates/s of c on (t, h, mk) -> o, CUDA events on our stream, max over ranks"""
            run_args = (ctx.h, p2z.C.byref(c), t.data_ptr(), h.data_ptr(), mk.data_ptr(), o.data_ptr(),
                        p2z.C.c_void_p(stream.cuda_stream), None)
            for _ in range(3):
                p2z.lib.p2z_run_device(*run_args)
            torch.cuda.synchronize()
            barrier(world)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            n = max(3, args.steps // 2)
            a.record(stream)
            for _ in range(n):
                p2z.lib.p2z_run_device(*run_args)
            b.record(stream)
            torch.cuda.synchronize()
            t_ms = barrier_max(world, a.elapsed_time(b)) / n
            return u_upd * world / (t_ms / 1e3)

        def cfg_for(sched):
            return p2z.make_config(bsize=32, nevts=len(counts), event_ntrks=counts, nlayer=20, schedule=sched,
                                   block_threads=blocks.get(sched, 32))

        for sched in ("persistent", "per_event"):
            res[sched] = timed(cfg_for(sched), udt, udh, udm, udo)
        # the launch shape the autotuner chose for this workload (schedule AUTO, block size and threads
        # per track open: the context applies the sweep's best, window sorting included)
        tuned_rate = None
        if tune_uneven is not None:
            tuned_rate = timed(p2z.make_config(bsize=32, nevts=len(counts), event_ntrks=counts, nlayer=20,
                                               schedule="auto", block_threads=0, threads_per_track=0),
                               udt, udh, udm, udo)
        # the same batched run with each 128-slot window in order of hit count (in-library sort)
        csw = cfg_for("persistent")
        csw.flags |= p2z.FLAG_SORT_WINDOWS
        res["persistent_sorted_windows"] = timed(csw, udt, udh, udm, udo)
        # the plain form as the reference's GPU build issues it: launches spread over 10 streams
        c10 = cfg_for("per_event")
        c10.flags |= p2z.FLAG_PER_EVENT_STREAMS
        res["per_event_10_streams"] = timed(c10, udt, udh, udm, udo)
        # the same sample with each event's tracks ordered by hit count (a packing choice of the caller)
        ts, hs, ms_, perm, util_packed, util_ordered = order_by_hits(torch, counts, udt, udh, udm)
        torch.cuda.synchronize()  # the copies are made on torch's stream; the runs read them on ours
        ordered = {}
        for sched in ("persistent", "flat"):
            ordered[sched] = timed(cfg_for(sched), ts, hs, ms_, udo)
        # same per-track results: the ordered run's outputs, put back in packed order, equal the packed run's
        uo = torch.empty_like(udo)
        ctx.run_device(cfg_for("persistent"), udt, udh, udo, d_mask=udm)
        ctx.run_device(cfg_for("persistent"), ts, hs, uo, d_mask=ms_)
        back = torch.empty_like(uo.permute(0, 2, 1).reshape(perm.numel(), -1))
        back[perm] = uo.permute(0, 2, 1).reshape(perm.numel(), -1)
        same = bool((back.view(torch.int32) == udo.permute(0, 2, 1).reshape(perm.numel(), -1).view(torch.int32)).all())
        # the same ordering done by the library (p2z_pack_by_hits_device): once per sample, then the passes
        # run on the packed copy and p2z_unpack_tracks_device puts each output back in the caller's order
        del back
        pt_, ph_, pm_ = torch.empty_like(udt), torch.empty_like(udh), torch.empty_like(udm)
        pperm = torch.empty(2 * unb * 32, dtype=torch.int64, device="cuda")
        pack_ms = []
        for _ in range(2):  # the first call also allocates the context's scratch
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ctx.pack_by_hits_device(ucfg, udt, udh, pt_, ph_, pperm, d_mask_in=udm, d_mask_out=pm_, stream=stream)
            pack_ms.append((time.perf_counter() - t0) * 1e3)  # synchronous call, host wall time
        packed_rate = timed(cfg_for("persistent"), pt_, ph_, pm_, uo)
        ctx.run_device(cfg_for("persistent"), pt_, ph_, uo, d_mask=pm_, stream=stream)
        ua, ub = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ub2 = torch.empty_like(uo)
        ua.record(stream)
        ctx.unpack_tracks_device(ucfg, pperm, uo, ub2, stream=stream)
        ub.record(stream)
        torch.cuda.synchronize()
        lib_pack = {"note": "p2z_pack_by_hits_device once, then passes on the packed copy (persistent graph), "
                            "p2z_unpack_tracks_device back to the caller's order",
                    "pack_ms_first_call": pack_ms[0], "pack_ms": pack_ms[1],
                    "pack_bytes": int(2 * (pt_.numel() + ph_.numel() + pm_.numel()) * 4),
                    "batched_persistent_graph": packed_rate,
                    "unpack_ms": ua.elapsed_time(ub),
                    "same_results_as_packed": bool((ub2.view(torch.int32) == udo.view(torch.int32)).all())}
        del pt_, ph_, pm_, pperm, ub2
        bvp = {"workload": f"{len(counts)} events, track counts log-normal (median 3000, sigma 1, clipped 50-30000), "
                           "5-20 hits/track, 10% layers dropped",
               "tracks": int(counts.sum()), "updates_per_step": u_upd,
               "batched_persistent_graph": res["persistent"], "plain_per_event_launch": res["per_event"],
               "plain_per_event_launch_10_streams": res["per_event_10_streams"],
               "batched_persistent_graph_sorted_windows": res["persistent_sorted_windows"],
               "batched_autotuned": ({"updates_per_s": tuned_rate,
                                      "shape": {k: tune_uneven["best_bsize32_aosoa"][k] for k in
                                                ("schedule", "block_threads", "threads_per_track", "sorted_windows")}}
                                     if tuned_rate else None),
               "lane_utilisation": {"stored_order": util_packed, "sorted_windows": window_util(udm, 128),
                                    "note": "present-hit lane-steps / (32 x warp steps); sorted_windows: each "
                                            "128-slot window in order of hit count (P2Z_FLAG_SORT_WINDOWS)"},
               "ratio": res["persistent"] / res["per_event"],
               "ratio_vs_10_streams": res["persistent"] / res["per_event_10_streams"],
               "batched_roofline": {
                   "fp32_tflops": FLOPS_PER_UPDATE * res["persistent"] / 1e12,
                   "fp32_frac": FLOPS_PER_UPDATE * res["persistent"] / 1e12 / fp32_peak_live,
                   "hbm_gbs": (BYTES_HIT_PER_UPDATE * res["persistent"] +
                               BYTES_TRACK * int(counts.sum()) * res["persistent"] / u_upd) / 1e9,
                   "hbm_frac": (BYTES_HIT_PER_UPDATE * res["persistent"] +
                                BYTES_TRACK * int(counts.sum()) * res["persistent"] / u_upd) / 1e9 /
                               measured_peaks()["hbm_gbs"],
                   "fp32_frac_reference_form": {
                       k: FLOPS_PER_UPDATE_REFERENCE_FORM * v / 1e12 / fp32_peak_live
                       for k, v in (("stored_order", res["persistent"]),
                                    ("sorted_windows", res["persistent_sorted_windows"]),
                                    ("ordered_by_hits", ordered["persistent"]),
                                    ("library_packing", lib_pack["batched_persistent_graph"]))},
                   "note": "present-hit updates; bytes = 24 per present hit + 228 per real track (in, out, mask); "
                           "fp32_frac_reference_form counts the update as the reference writes it"},
               "block_threads": blocks,
               "ordered_by_hits": {"note": "same events, each event's tracks packed in order of hit count",
                                   "batched_persistent_graph": ordered["persistent"],
                                   "flat": ordered["flat"], "ratio_vs_plain": ordered["persistent"] / res["per_event"],
                                   "lane_utilisation_as_packed": util_packed,
                                   "lane_utilisation_ordered": util_ordered,
                                   "same_results_as_packed": same},
               "library_packing": lib_pack,
               "autotune": tune_uneven}
        del udt, udh, udo, udm, ts, hs, ms_, uo

    # serving: continuous batching under Poisson arrivals
    serving = None
    if not args.no_serving:
        serving = run_serving(p2z, local, rank, args)

    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return 0

    peaks = measured_peaks()
    launch_ms = ms_step / max(1, launches_per_step)
    achieved_gbs = BYTES_PER_UPDATE * updates / launches_per_step / (launch_ms / 1e3) / 1e9
    tpu = profile_traffic_per_update()
    sm_max = clk["sm_max_mhz"] or 1965.0
    fp32_nominal = 148 * FP32_LANES_PER_SM * 2 * sm_max * 1e6 / 1e12
    fp32_peak = fp32_peak_live
    fp32_ach = FLOPS_PER_UPDATE * updates / (launch_ms / 1e3) / 1e12
    line = {
        "metric": METRIC, "value": value, "unit": "updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(nev, world),
        "form": ("precise (default; no FP64 instruction)" if args.update == "v2" else f"update kind {args.update}"),
        "launch": launch,
        "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved_gbs / peaks["hbm_gbs"],
                     "traffic": (tpu * updates / launches_per_step) if tpu else None,
                     "peak_source": peaks["source"] + " (MEASURED_PEAKS.json hbm_gbs, burst copy)",
                     "bytes_per_update": BYTES_PER_UPDATE},
        "fp32_roofline": {"achieved": fp32_ach, "peak": fp32_peak, "unit": "TFLOP/s", "frac": fp32_ach / fp32_peak,
                          "flops_per_update": FLOPS_PER_UPDATE,
                          "peak_source": "measured in this run (p2z_measure_peaks): independent FMA chains on "
                                         "every lane of every SM, the faster of scalar FFMA "
                                         f"({live_peaks['fp32_ffma_tflops']:.1f}) and paired FFMA2 "
                                         f"({live_peaks['fp32_ffma2_tflops']:.1f} TFLOP/s)",
                          "nominal": fp32_nominal,
                          "reference_form": {
                              "flops_per_update": FLOPS_PER_UPDATE_REFERENCE_FORM,
                              "frac": FLOPS_PER_UPDATE_REFERENCE_FORM * updates / (launch_ms / 1e3) / 1e12 / fp32_peak,
                              "note": "the update counted as the reference writes it, products with the "
                                      "Jacobian's known zeros included; this kernel does not execute those"}},
        "clocks": clk,
        "measured_peaks": live_peaks,
        "autotune": tune_head,
        "threads_per_track": lanes,
        "gpu_launches": launches_per_step * args.steps,
        "e2e": e2e,
        "batched_vs_plain": bvp,
        "reference_gpu": ref_gpu,
        "serving": serving,
        "outputs_finite": out_ok,
    }
    if cpu_sample is not None:
        line["cpu_baseline"] = cpu_baseline(p2z, *cpu_sample)
    print(json.dumps(line))
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
