"""Host side of the boundary: the library loads and exports every declared
symbol, the reference-compatible input preparation, the validation block, the
physics generator and layer masks, argument checking.  CPU only."""
import ctypes
import json
import subprocess
import sys

import numpy as np
import pytest

from conftest import GOLDEN, ROOT


def test_library_exports_every_declared_symbol(p2z):
    names = p2z.declared_symbols()
    assert len(names) >= 20
    lib = ctypes.CDLL(str(p2z.LIB_PATH))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


@pytest.mark.parametrize("lang", ["c", "c++"])
@pytest.mark.parametrize("bsize", [8, 32])
def test_c_abi_after_the_reference_macros(tmp_path, lang, bsize):
    """p2z.h included after the reference's size macros, as a maintainer adds
    it to the OpenMP source; the config filled by p2z_config_init from those
    macros; the macros intact after the header.  Compiled as C and as C++."""
    exe = tmp_path / "c_abi_macros"
    cc = ["gcc", "-std=c11"] if lang == "c" else ["g++", "-std=c++17", "-x", "c++"]
    pkg = ROOT / "p2z-tests_b200"
    cmd = [*cc, "-O2", "-Wall", "-Werror", f"-I{ROOT / 'include'}", f"-Dbsize={bsize}",
           str(ROOT / "tests" / "cpp" / "c_abi_macros.c"), "-x", "none", "-o", str(exe), f"-L{pkg}", "-lp2z",
           f"-Wl,-rpath,{pkg}"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    lines = r.stdout.splitlines()
    assert lines[0] == "abi_version 2"
    assert lines[1] == f"sizes {bsize} 100 9600 20"
    assert lines[2] == "niter 5 update 0 schedule 0 block 0 flags 0 layout 0 tpt 0 kfact 0 event_ntrks 0"
    assert lines[3] == f"batches {100 * 9600 // bsize}"


def test_version_and_sizes(p2z):
    assert p2z.lib.p2z_version(None, 0) == p2z.ABI_VERSION
    assert "sm_100a" in p2z.version()
    for b in (8, 16, 32, 64):
        assert p2z.lib.p2z_sizeof_mptrk(b) == 28 * b * 4
        assert p2z.lib.p2z_sizeof_mphit(b) == 9 * b * 4
    assert p2z.lib.p2z_sizeof_mptrk(12) == 0


@pytest.mark.parametrize("bsize", [8, 16, 32, 64])
def test_prepare_bit_exact_vs_reference(p2z, oracle, kat_seed, bsize):
    """srand(1) + prepareTracks + prepareHits of the reference, bit for bit (2 x 128 tracks)."""
    if not oracle.ref_available(f"b{bsize}"):
        pytest.skip("reference build absent")
    rt, rh = oracle.ref_prepare(f"b{bsize}", *kat_seed)
    mt, mh = p2z.prepare(p2z.make_atrk(*kat_seed[0]), p2z.make_ahits(kat_seed[1]), bsize, 2, 128, 20)
    assert np.array_equal(rt.view(np.uint32), mt.view(np.uint32))
    assert np.array_equal(rh.view(np.uint32), mh.view(np.uint32))


def test_prepare_rejects_too_few_hits(p2z, kat_seed):
    with pytest.raises(p2z.P2zError):
        p2z.prepare(p2z.make_atrk(*kat_seed[0]), p2z.make_ahits(kat_seed[1][:10]), 32, 1, 32, 20)


def test_prepare_does_not_touch_global_rand(p2z, kat_seed):
    libc = ctypes.CDLL(None)
    libc.srand(123)
    a = libc.rand()
    libc.srand(123)
    p2z.prepare(p2z.make_atrk(*kat_seed[0]), p2z.make_ahits(kat_seed[1]), 32, 1, 32, 20)
    assert libc.rand() == a


def test_validation_block_matches_reference_printout(p2z, oracle, kat_seed):
    """p2z_validate/p2z_print_validation print the reference's block for the
    reference's own outputs (2 x 128 tracks of the known-answer input)."""
    gold = np.load(GOLDEN / "ref_kat_small.npz")["out_fma"]
    v = p2z.validate(gold, 32, 2, 128, kat_seed[1][19][0])
    assert v.nnans == 0 and v.nfail == 0 and v.ngood == 256
    code = f"""
import sys, numpy as np
sys.path.insert(0, {str(ROOT / 'tests')!r})
import conftest
p2z = conftest.load_p2z()
gold = np.load({str(GOLDEN / 'ref_kat_small.npz')!r})['out_fma']
seed = conftest.read_seed({str(GOLDEN / 'kat_seed.txt')!r})
p2z.print_validation(p2z.validate(gold, 32, 2, 128, seed[1][19][0]))
"""
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120).stdout
    lines = out.strip().splitlines()
    assert lines[0].startswith("track x avg=") and lines[-1].startswith("number of tracks failed=0")
    assert len(lines) == 11
    # the same accumulations done independently in numpy
    a = p2z.tracks_to_aos(gold)
    x = a["par"][:, 0].astype(np.float64)
    assert lines[0].split()[2] == "avg=%f" % x.mean()


def test_validation_counts_nans_and_window(p2z):
    trk = p2z.empty_tracks(1, 8)
    trk[0, 0, :] = 18.5        # x near the last seed hit
    trk[0, 1, :] = 79.8
    trk[0, 2, :] = -80.5
    trk[0, 3, :] = 1 / 12.0    # pt 12
    trk[0, 4, :] = 1.3
    trk[0, 5, :] = 2.8
    trk[0, 0, 0] = np.nan
    trk[0, 4, 1] = 10.0        # phi outside the window
    v = p2z.validate(trk, 8, 1, 8, [18.5, 79.8, -80.5])
    assert v.nnans == 1 and v.nfail == 1 and v.ngood == 6


def test_formatted_line(p2z):
    code = f"""
import sys
sys.path.insert(0, {str(ROOT / 'tests')!r})
import conftest
p2z = conftest.load_p2z()
p2z.lib.p2z_print_formatted(5, 10, 9600, 32, 0.25, 1.5, 16)
"""
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=60).stdout
    # field order of the reference's line, read positionally by tools/compare.py:12
    assert out.strip() == "formatted 5 10 9600 32 300 0.250000 0 1.500000 16"


def test_config_validation(p2z):
    assert p2z.num_batches(p2z.make_config(bsize=32, nevts=10, ntrks=9600)) == 3000
    assert p2z.num_batches(p2z.make_config(bsize=8, nevts=3, event_ntrks=[1, 8, 9])) == 1 + 1 + 2
    for bad in [dict(bsize=12), dict(nlayer=0), dict(nlayer=33), dict(ntrks=33), dict(update=9),
                dict(schedule=7), dict(block_threads=48), dict(nevts=-1)]:
        kw = dict(bsize=32, nevts=1, ntrks=32)
        kw.update(bad)
        cfg = p2z.make_config(**kw)
        assert p2z.lib.p2z_num_batches(ctypes.byref(cfg)) == -1, bad
    cfg = p2z.make_config()
    cfg.abi_version = 99
    assert p2z.lib.p2z_num_batches(ctypes.byref(cfg)) == -1


def test_physics_generator_is_deterministic_and_on_helix(p2z, oracle):
    cfg = p2z.make_config(bsize=16, nevts=2, ntrks=64, nlayer=20)
    t1, h1 = p2z.generate_physics(cfg, p2z.physics_params(nthreads=1))
    t2, h2 = p2z.generate_physics(cfg, p2z.physics_params(nthreads=7))
    assert np.array_equal(t1.view(np.uint32), t2.view(np.uint32)) and np.array_equal(h1, h2)
    a = p2z.tracks_to_aos(t1)
    hh = p2z.hits_to_aos(h1)
    assert set(np.unique(a["q"])) <= {-1, 1}
    pt = 1 / a["par"][:, 3]
    assert pt.min() > 0.45 and pt.max() < 22
    eta = -np.log(np.tan(a["par"][:, 5] / 2))
    assert eta.min() > 1.55 and eta.max() < 2.55
    z = hh["pos"][:, :, 2]
    assert np.allclose(z[:, 0], 30, atol=1e-3) and np.allclose(z[:, -1], 270, atol=1e-3)
    # covariances are positive definite
    for i in range(0, 128, 17):
        C = np.zeros((6, 6))
        for r in range(6):
            for c in range(r + 1):
                C[r, c] = C[c, r] = a["cov"][i, r * (r + 1) // 2 + c]
        assert np.linalg.eigvalsh(C).min() > 0
    # the FP64 filter ends close to the last hit (hits lie on the helix)
    o = oracle.run_f64(t1, h1)
    d = np.hypot(o[:, 0] - hh["pos"][:, -1, 0], o[:, 1] - hh["pos"][:, -1, 1])
    assert np.median(d) < 0.01


def test_uneven_generator_and_masks(p2z):
    counts = np.array([5, 0, 17, 32], dtype=np.int64)
    cfg = p2z.make_config(bsize=16, nevts=4, event_ntrks=counts, nlayer=20)
    nb = p2z.num_batches(cfg)
    assert nb == 1 + 0 + 2 + 2
    t, h, m = p2z.generate_physics(cfg, with_mask=True)
    real = np.zeros(nb * 16, bool)
    real[0:5] = True
    real[16:16 + 17] = True
    real[48:48 + 32] = True
    assert np.array_equal(m != 0, real)
    p2z.mask_layers(m, 20, min_hits=5, max_hits=20, drop_prob=0.1, seed=3)
    pc = np.array([bin(int(x)).count("1") for x in m])
    assert (pc[real] >= 5).all() and (pc[real] <= 20).all() and (pc[~real] == 0).all()
    assert 0.05 < 1 - pc[real].sum() / sum(int(x).bit_length() for x in m[real]) < 0.2


def test_driver_prints_reference_lines_without_gpu(p2z):
    """p2z_main parses its seed file and fails cleanly when no GPU is present."""
    exe = ROOT / "p2z-tests_b200" / "p2z_main"
    if not exe.exists():
        pytest.skip("driver not built")
    r = subprocess.run([str(exe), str(GOLDEN / "kat_seed.txt"), "1", "32", "32", "20", "1"],
                       capture_output=True, text=True, timeout=120)
    assert "track in pos: x=20.048365" in r.stdout
    assert "hit in layer=19, pos: x=7.320264, y=27.722622, z=-80.523956" in r.stdout


def test_dump_tracks_writes_the_selected_tracks(p2z, tmp_path):
    """DUMP_OUTPUT files: one "%f" line per track passing the validation's
    NaN test and window, output coordinates and input coordinates."""
    trk_in = p2z.empty_tracks(1, 8)
    trk_in[0, :3, :] = np.arange(24, dtype=np.float32).reshape(3, 8)
    out = p2z.empty_tracks(1, 8)
    out[0, 0, :] = 18.5
    out[0, 1, :] = 79.8
    out[0, 2, :] = -80.5
    out[0, 3, :] = 1 / 12.0
    out[0, 4, :] = 1.3
    out[0, 5, :] = 2.8
    out[0, 0, 2] = np.nan      # dropped: not finite
    out[0, 5, 5] = 9.0         # dropped: theta outside the window
    out[0, 0, 7] = 18.25
    p2z.dump_tracks(trk_in, out, 8, 1, 8, [18.5, 79.8, -80.5], tmp_path)
    kept = [0, 1, 3, 4, 6, 7]
    ox = (tmp_path / "output_x.txt").read_text().split()
    assert ox == ["%f" % v for v in out[0, 0, kept].astype(np.float64)]
    for name, row in (("input_x.txt", 0), ("input_y.txt", 1), ("input_z.txt", 2)):
        assert (tmp_path / name).read_text().split() == ["%f" % v for v in trk_in[0, row, kept].astype(np.float64)]
    assert len((tmp_path / "output_z.txt").read_text().split()) == len(kept)


def test_device_call_stream_selection(p2z):
    """The binding's choice of stream for a device call: an explicit stream
    (handle or object with .cuda_stream) as given, the legacy default stream's
    handle 0 as cudaStreamLegacy (NULL means the context's own stream in the
    C ABI), and no stream for arguments that are not torch CUDA tensors."""
    class FakeStream:
        def __init__(self, h):
            self.cuda_stream = h
    assert p2z._stream(0) == p2z.CUDA_STREAM_LEGACY
    assert p2z._stream(0x7f00) == 0x7f00
    assert p2z._stream(FakeStream(0)) == p2z.CUDA_STREAM_LEGACY
    assert p2z._stream(FakeStream(0x5000)) == 0x5000
    assert p2z._stream(None, np.zeros(4, np.float32), 12345, None) is None
    import torch
    assert p2z._stream(None, torch.zeros(4)) is None  # a CPU tensor


def test_server_refuses_flags_it_cannot_honour(p2z):
    """The server's group launches honour the accurate-trigonometry,
    reference-rounding and full-hit flags only; strict mode and the input
    scan (no per-request status) and the schedule flags are refused before
    any device is touched."""
    for fl in (p2z.FLAG_STRICT, p2z.FLAG_CHECK_INPUTS, p2z.FLAG_SORT_WINDOWS, p2z.FLAG_NO_GRAPH,
               p2z.FLAG_PER_EVENT_STREAMS):
        with pytest.raises(p2z.P2zError) as e:
            p2z.Server(bsize=32, nlayer=20, flags=fl | p2z.FLAG_ACCURATE_TRIG)
        assert e.value.status == p2z.UNSUPPORTED, fl
    with pytest.raises(p2z.P2zError) as e:
        p2z.Server(bsize=32, nlayer=20, update="3x3_f64", flags=p2z.FLAG_REFERENCE_ROUNDING)
    assert e.value.status == p2z.UNSUPPORTED
    for kw in (dict(kfact=float("nan")), dict(block_threads=48), dict(block_threads=512)):
        with pytest.raises(p2z.P2zError) as e:
            p2z.Server(bsize=32, nlayer=20, **kw)
        assert e.value.status == p2z.BAD_ARG, kw


def test_unknown_flag_bits_are_refused(p2z):
    """A config with a flag bit no P2Z_FLAG_* defines is refused (P2Z_BAD_ARG)
    rather than run with the bit ignored: by the config checks every entry
    point shares (here through p2z_num_batches) and by the allocation-free
    entry point."""
    cfg = p2z.make_config(bsize=32, nevts=1, ntrks=64, nlayer=20, flags=0x100)
    assert p2z.lib.p2z_num_batches(p2z.C.byref(cfg)) == -1
    assert "unknown flag bits" in p2z.lib.p2z_last_error(None).decode()
    cfg.flags = p2z.FLAG_ACCURATE_TRIG
    assert p2z.lib.p2z_num_batches(p2z.C.byref(cfg)) == 2
    cfg.flags = 0x80000000
    rc = p2z.lib.p2z_run_device_noalloc(p2z.C.byref(cfg), None, None, None, None, None)
    assert rc == p2z.BAD_ARG
    assert "unknown flag bits" in p2z.lib.p2z_last_error(None).decode()


def test_niter_and_kfact_are_checked(p2z):
    cfg = p2z.make_config(bsize=32, nevts=1, ntrks=64, nlayer=20, niter=-1)
    assert p2z.lib.p2z_num_batches(p2z.C.byref(cfg)) == -1
    cfg.niter = 0
    assert p2z.lib.p2z_num_batches(p2z.C.byref(cfg)) == 2
    for k in (float("nan"), float("inf")):
        cfg.kfact = k
        assert p2z.lib.p2z_num_batches(p2z.C.byref(cfg)) == -1
        assert "kfact" in p2z.lib.p2z_last_error(None).decode()
        assert p2z.lib.p2z_run_device_noalloc(p2z.C.byref(cfg), None, None, None, None, None) == p2z.BAD_ARG
