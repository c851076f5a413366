"""Multi-process host logic of the sharded (one GPU per process) form, run as
world-size-2 gloo ranks on CPU: event sharding, the validation block reduced
across shards, and a rank that dies before the collective."""
import json
import multiprocessing as mp
import os
import pathlib
import socket
import sys

import numpy as np
import pytest

from conftest import GOLDEN, ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, outdir, mode):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, str(ROOT / "tests"))
    import datetime

    import torch
    import torch.distributed as dist
    import conftest
    p2z = conftest.load_p2z()
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    out = np.load(GOLDEN / "ref_kat_small.npz")["out_fma"]          # 2 events x 128 tracks
    seed = conftest.read_seed(GOLDEN / "kat_seed.txt")
    e0, e1 = p2z.shard_events([128, 128], world)[rank]
    nb_ev = 128 // 32
    shard = np.ascontiguousarray(out[e0 * nb_ev:e1 * nb_ev])

    def allreduce(a):
        t = torch.from_numpy(a)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        a[:] = t.numpy()

    result = {}
    try:
        if mode == "die" and rank == 1:
            os._exit(3)  # leaves between steps, no collective in flight
        v = p2z.validate_sharded(shard, 32, e1 - e0, 128, seed[1][19][0], allreduce=allreduce)
        result = {"ok": True, "v": v.as_dict()}
    except Exception as exc:  # the survivor learns of the dead peer from the collective
        result = {"ok": False, "error": type(exc).__name__}
    (pathlib.Path(outdir) / f"rank{rank}.json").write_text(json.dumps(result))
    try:
        dist.destroy_process_group()
    except Exception:
        pass


def _spawn(world, mode, tmp_path):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path), mode)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        if p.is_alive():
            p.kill()
            p.join()
    return procs


def test_shard_events_balances_tracks(p2z):
    assert p2z.shard_events([9600] * 1000, 4) == [(0, 250), (250, 500), (500, 750), (750, 1000)]
    counts = np.array([50, 30000, 3000, 3000, 100, 8000, 9000, 70])
    sh = p2z.shard_events(counts, 3)
    assert sh[0][0] == 0 and sh[-1][1] == len(counts)
    assert all(a[1] == b[0] for a, b in zip(sh, sh[1:]))
    loads = [counts[a:b].sum() for a, b in sh]
    assert max(loads) <= counts.max() + counts.sum() / 3


def test_sharded_validation_equals_single_process(p2z, kat_seed, tmp_path):
    procs = _spawn(2, "ok", tmp_path)
    assert all(p.exitcode == 0 for p in procs)
    r = [json.loads((tmp_path / f"rank{i}.json").read_text()) for i in range(2)]
    assert r[0]["ok"] and r[1]["ok"]
    out = np.load(GOLDEN / "ref_kat_small.npz")["out_fma"]
    single = p2z.validate(out, 32, 2, 128, kat_seed[1][19][0]).as_dict()
    for k, v in single.items():
        assert r[0]["v"][k] == pytest.approx(v, rel=1e-12, abs=1e-15), k
        assert r[1]["v"][k] == r[0]["v"][k]


def test_dead_rank_is_detected_by_survivor(tmp_path):
    procs = _spawn(2, "die", tmp_path)
    assert procs[1].exitcode == 3
    assert procs[0].exitcode == 0
    r0 = json.loads((tmp_path / "rank0.json").read_text())
    assert r0["ok"] is False
