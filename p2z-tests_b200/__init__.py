"""Python binding of libp2z.so, the B200 propagate-to-z + Kalman-update library.

The product is the shared library built from ``csrc/`` (sm_100a kernels and the
``extern "C"`` boundary declared in ``include/p2z.h``).  This module only binds
that C ABI with ctypes for tests, benchmarks and Python callers; it has no
compute path of its own.  Importing it fails loudly when the library has not
been built -- there is no fallback.

Layout helpers use numpy views of the reference's AOSOA structs
(src/propagate-toz-test_OMP.cpp:57-125): a track batch of width B is
``par[6*B] cov[21*B] q[B]`` (28*B 32-bit words), a hit batch ``pos[3*B] cov[6*B]``.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib

import numpy as np

PKG_DIR = pathlib.Path(__file__).resolve().parent
# P2Z_LIBRARY selects another build of the same library (e.g. a tuning variant).
LIB_PATH = pathlib.Path(os.environ.get("P2Z_LIBRARY", PKG_DIR / "libp2z.so"))
INCLUDE_H = PKG_DIR.parent / "include" / "p2z.h"

ABI_VERSION = 2
KFACT_DEFAULT = np.float32(100.0 / (-0.299792458 * 3.8112))
TRK_WORDS = 28
HIT_WORDS = 9

# status codes
OK, BAD_ARG, OOM, NONFINITE_INPUT, SINGULAR, TIMEOUT, CUDA_ERROR, NO_DEVICE, UNSUPPORTED, NOT_READY = range(10)
STATUS_NAMES = ["OK", "BAD_ARG", "OOM", "NONFINITE_INPUT", "SINGULAR", "TIMEOUT", "CUDA_ERROR", "NO_DEVICE",
                "UNSUPPORTED", "NOT_READY"]
# update kinds
UPDATE_V2, UPDATE_V2_COMP, UPDATE_3X3_F64, UPDATE_3X3_COMP, UPDATE_F64 = range(5)
UPDATE_NAMES = {"v2": UPDATE_V2, "v2_comp": UPDATE_V2_COMP, "3x3_f64": UPDATE_3X3_F64,
                "3x3_comp": UPDATE_3X3_COMP, "f64": UPDATE_F64}
# schedules
SCHED_AUTO, SCHED_FLAT, SCHED_PER_EVENT, SCHED_PERSISTENT, SCHED_STAGED = range(5)
SCHED_NAMES = {"auto": SCHED_AUTO, "flat": SCHED_FLAT, "per_event": SCHED_PER_EVENT,
               "persistent": SCHED_PERSISTENT, "staged": SCHED_STAGED}
SCHED_LABELS = {v: k for k, v in SCHED_NAMES.items()}
# array layouts
LAYOUT_AOSOA, LAYOUT_SOA = 0, 1
LAYOUT_NAMES = {"aosoa": LAYOUT_AOSOA, "soa": LAYOUT_SOA}
LAYOUT_LABELS = {v: k for k, v in LAYOUT_NAMES.items()}
# flags
FLAG_CHECK_INPUTS = 0x1
FLAG_STRICT = 0x2
FLAG_NO_GRAPH = 0x4
FLAG_ACCURATE_TRIG = 0x8
FLAG_FULL_HITS = 0x10
FLAG_REFERENCE_ROUNDING = 0x20
FLAG_PER_EVENT_STREAMS = 0x40
FLAG_SORT_WINDOWS = 0x80


class P2zError(RuntimeError):
    def __init__(self, status: int, msg: str):
        name = STATUS_NAMES[status] if 0 <= status < len(STATUS_NAMES) else str(status)
        super().__init__(f"p2z {name}: {msg}")
        self.status = status


class Config(C.Structure):
    _fields_ = [("abi_version", C.c_int32), ("bsize", C.c_int32), ("nevts", C.c_int64), ("ntrks", C.c_int64),
                ("nlayer", C.c_int32), ("niter", C.c_int32), ("kfact", C.c_float), ("update", C.c_int32),
                ("schedule", C.c_int32), ("block_threads", C.c_int32), ("flags", C.c_uint32),
                ("layout", C.c_int32), ("event_ntrks", C.POINTER(C.c_int64)), ("threads_per_track", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("kernel_ms", C.c_double), ("h2d_ms", C.c_double), ("d2h_ms", C.c_double),
                ("total_ms", C.c_double), ("track_slots", C.c_int64), ("updates", C.c_int64),
                ("h2d_bytes", C.c_int64), ("d2h_bytes", C.c_int64), ("launches", C.c_int32),
                ("singular", C.c_int32)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class Atrk(C.Structure):
    _fields_ = [("par", C.c_float * 6), ("cov", C.c_float * 21), ("q", C.c_int32)]


class Ahit(C.Structure):
    _fields_ = [("pos", C.c_float * 3), ("cov", C.c_float * 6)]


class PhysicsParams(C.Structure):
    _fields_ = [("seed", C.c_uint64)] + [(n, C.c_double) for n in (
        "pt_min", "pt_max", "eta_min", "eta_max", "sigma_vz", "sig_xy", "sig_z", "rel_sig_ipt", "sig_phi",
        "sig_theta", "rho_max", "z_first", "z_last", "hit_sig_xy", "hit_sig_z")] + [
        ("kfact", C.c_float), ("nthreads", C.c_int32)]


class Validation(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("avgx", "avgy", "avgz", "avgdx", "avgdy", "avgdz", "avgpt", "avgphi",
                                          "avgtheta", "stdx", "stdy", "stdz", "stddx", "stddy", "stddz")] + [
        ("nnans", C.c_int64), ("nfail", C.c_int64), ("ngood", C.c_int64)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class ValidationPartial(C.Structure):
    _fields_ = [("sum", C.c_double * 9), ("sq", C.c_double * 6), ("nnans", C.c_int64), ("nfail", C.c_int64),
                ("ngood", C.c_int64)]

    def to_array(self) -> np.ndarray:
        """Doubles and counts as one float64 vector (for an all-reduce)."""
        return np.array(list(self.sum) + list(self.sq) + [self.nnans, self.nfail, self.ngood], dtype=np.float64)

    @classmethod
    def from_array(cls, a):
        p = cls()
        p.sum[:] = [float(x) for x in a[:9]]
        p.sq[:] = [float(x) for x in a[9:15]]
        p.nnans, p.nfail, p.ngood = (int(round(x)) for x in a[15:18])
        return p


class TuneEntry(C.Structure):
    _fields_ = [("bsize", C.c_int32), ("layout", C.c_int32), ("schedule", C.c_int32), ("block_threads", C.c_int32),
                ("threads_per_track", C.c_int32), ("flags", C.c_uint32), ("ms", C.c_double),
                ("updates_per_s", C.c_double)]

    def as_dict(self):
        d = {n: getattr(self, n) for n, _ in self._fields_}
        d["layout"] = LAYOUT_LABELS.get(d["layout"], d["layout"])
        d["schedule"] = SCHED_LABELS.get(d["schedule"], d["schedule"])
        d["sorted_windows"] = bool(d.pop("flags") & FLAG_SORT_WINDOWS)
        return d


class ServerConfig(C.Structure):
    _fields_ = [("abi_version", C.c_int32), ("bsize", C.c_int32), ("nlayer", C.c_int32), ("update", C.c_int32),
                ("flags", C.c_uint32), ("kfact", C.c_float), ("device_budget_bytes", C.c_int64),
                ("max_inflight", C.c_int32), ("block_threads", C.c_int32)]


class RequestInfo(C.Structure):
    _fields_ = [("submit_s", C.c_double), ("admit_s", C.c_double), ("launch_s", C.c_double),
                ("done_s", C.c_double), ("ntrks", C.c_int64), ("updates", C.c_int64), ("group_events", C.c_int32),
                ("status", C.c_int32)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class Peaks(C.Structure):
    _fields_ = [("fp32_ffma_tflops", C.c_double), ("fp32_ffma2_tflops", C.c_double), ("h2d_gbs", C.c_double),
                ("d2h_gbs", C.c_double), ("bidir_gbs", C.c_double), ("copy_bytes", C.c_int64), ("sms", C.c_int32)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


# Every symbol include/p2z.h declares, with its ctypes signature.
_VP, _CVP = C.c_void_p, C.c_void_p
_SIGS = {
    "p2z_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "p2z_destroy": (C.c_int, [_VP]),
    "p2z_status_string": (C.c_char_p, [C.c_int]),
    "p2z_last_error": (C.c_char_p, [_VP]),
    "p2z_version": (C.c_int, [C.c_char_p, C.c_size_t]),
    "p2z_num_batches": (C.c_int64, [C.POINTER(Config)]),
    "p2z_sizeof_mptrk": (C.c_size_t, [C.c_int]),
    "p2z_sizeof_mphit": (C.c_size_t, [C.c_int]),
    "p2z_run": (C.c_int, [_VP, C.POINTER(Config), _CVP, _CVP, _CVP, _VP, C.POINTER(Stats)]),
    "p2z_run_device": (C.c_int, [_VP, C.POINTER(Config), _CVP, _CVP, _CVP, _VP, _VP, C.POINTER(Stats)]),
    "p2z_run_device_noalloc": (C.c_int, [C.POINTER(Config), _CVP, _CVP, _CVP, _VP, _VP]),
    "p2z_step_device": (C.c_int, [_VP, C.c_int, C.c_int64, _VP, _CVP, C.c_int, C.c_int, C.c_int, C.c_int,
                                  C.c_float]),
    "p2z_prepare": (C.c_int, [C.POINTER(Atrk), C.POINTER(Ahit), C.c_int, C.c_int, C.c_int64, C.c_int64, C.c_int,
                              C.c_double, C.c_double, _VP, _VP]),
    "p2z_prepare_device": (C.c_int, [_VP, C.POINTER(Atrk), C.POINTER(Ahit), C.c_int, C.c_int, C.c_int64, C.c_int64,
                                     C.c_int, C.c_double, C.c_double, _VP, _VP, _VP]),
    "p2z_physics_defaults": (None, [C.POINTER(PhysicsParams)]),
    "p2z_generate_physics": (C.c_int, [C.POINTER(PhysicsParams), C.POINTER(Config), _VP, _VP, _VP]),
    "p2z_mask_layers": (C.c_int, [_VP, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_double, C.c_uint64]),
    "p2z_generate_physics_device": (C.c_int, [_VP, C.POINTER(PhysicsParams), C.POINTER(Config), _VP, _VP, _VP, _VP]),
    "p2z_mask_layers_device": (C.c_int, [_VP, _VP, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_double, C.c_uint64,
                                         _VP]),
    "p2z_validate": (C.c_int, [_CVP, C.c_int, C.c_int64, C.c_int64, C.POINTER(C.c_float), C.POINTER(Validation)]),
    "p2z_validate_partial": (C.c_int, [_CVP, C.c_int, C.c_int64, C.c_int64, C.POINTER(C.c_float),
                                       C.POINTER(C.c_double), C.POINTER(ValidationPartial)]),
    "p2z_validate_means": (None, [C.POINTER(ValidationPartial), C.POINTER(C.c_double)]),
    "p2z_validate_combine": (C.c_int, [C.POINTER(ValidationPartial), C.POINTER(ValidationPartial),
                                       C.POINTER(Validation)]),
    "p2z_validate_device": (C.c_int, [_VP, _CVP, C.c_int, C.c_int64, C.c_int64, C.POINTER(C.c_float),
                                      C.POINTER(Validation), _VP]),
    "p2z_validate_partial_device": (C.c_int, [_VP, _CVP, C.c_int, C.c_int64, C.c_int64, C.POINTER(C.c_float),
                                              C.POINTER(C.c_double), C.POINTER(ValidationPartial), _VP]),
    "p2z_print_validation": (None, [C.POINTER(Validation)]),
    "p2z_dump_tracks": (C.c_int, [_CVP, _CVP, C.c_int, C.c_int64, C.c_int64, C.POINTER(C.c_float), C.c_char_p]),
    "p2z_print_formatted": (None, [C.c_int, C.c_int64, C.c_int64, C.c_int, C.c_double, C.c_double, C.c_int]),
    "p2z_server_create": (C.c_int, [C.c_int, C.POINTER(ServerConfig), C.POINTER(C.c_void_p)]),
    "p2z_server_destroy": (C.c_int, [_VP]),
    "p2z_server_submit": (C.c_int, [_VP, _CVP, _CVP, _CVP, C.c_int64, _VP, C.POINTER(C.c_int64)]),
    "p2z_server_poll": (C.c_int, [_VP, C.c_int64, C.POINTER(RequestInfo)]),
    "p2z_server_wait": (C.c_int, [_VP, C.c_int64, C.c_double, C.POINTER(RequestInfo)]),
    "p2z_server_now": (C.c_double, [_VP]),
    "p2z_server_replay": (C.c_int, [_VP, C.c_int64, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                    C.POINTER(C.c_void_p), C.POINTER(C.c_int64), C.POINTER(C.c_void_p),
                                    C.POINTER(C.c_double), C.POINTER(RequestInfo)]),
    "p2z_relayout_device": (C.c_int, [_VP, C.POINTER(Config), C.POINTER(Config), _CVP, _CVP, _CVP, _VP, _VP, _VP,
                                      _VP]),
    "p2z_pack_by_hits_device": (C.c_int, [_VP, C.POINTER(Config), _CVP, _CVP, _CVP, _VP, _VP, _VP, _VP, _VP]),
    "p2z_unpack_tracks_device": (C.c_int, [_VP, C.POINTER(Config), _CVP, _CVP, _VP, _VP]),
    "p2z_autotune": (C.c_int, [_VP, C.POINTER(Config), _CVP, _CVP, _CVP, C.c_int, C.POINTER(TuneEntry), C.c_int,
                               C.POINTER(C.c_int), C.POINTER(TuneEntry)]),
    "p2z_measure_peaks": (C.c_int, [C.c_int, C.c_size_t, C.c_int, C.POINTER(Peaks)]),
    "p2z_host_alloc": (C.c_int, [C.POINTER(C.c_void_p), C.c_size_t]),
    "p2z_device_alloc": (C.c_int, [_VP, C.POINTER(C.c_void_p), C.c_size_t]),
    "p2z_device_free": (C.c_int, [_VP, _VP]),
    "p2z_copy": (C.c_int, [_VP, _VP, _CVP, C.c_size_t]),
    "p2z_ref_rng_seed": (None, [_VP, C.c_uint32]),
    "p2z_ref_rng_rand": (C.c_int32, [_VP]),
    "p2z_ref_rng_randn": (C.c_float, [_VP]),
    "p2z_prepare_tracks": (C.c_int, [_VP, C.POINTER(Atrk), C.c_int, C.c_int64, C.c_int64, C.c_double, C.c_double,
                                     _VP]),
    "p2z_prepare_hits": (C.c_int, [_VP, C.POINTER(Ahit), C.c_int, C.c_int, C.c_int64, C.c_int64, C.c_int,
                                   C.c_double, _VP]),
    "p2z_host_free": (C.c_int, [_VP]),
}


def _load():
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is not built; run `make -C {PKG_DIR}` or __graft_entry__.build()")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def declared_symbols() -> list[str]:
    """Function names declared in include/p2z.h (parsed from the header)."""
    import re
    text = INCLUDE_H.read_text()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)  # comments are not declarations
    text = re.sub(r"//[^\n]*", " ", text)
    return sorted(set(re.findall(r"\b(p2z_[a-z0-9_]+)\s*\(", text)))


def _check(status: int, ctx=None):
    if status != OK:
        msg = lib.p2z_last_error(ctx)
        raise P2zError(status, (msg or b"").decode())


def measure_peaks(device=-1, copy_bytes=0, reps=0) -> dict:
    """FP32 FMA throughput (TFLOP/s) and pinned copy rates (GB/s) of the GPU
    (p2z_measure_peaks)."""
    pk = Peaks()
    _check(lib.p2z_measure_peaks(device, copy_bytes, reps, C.byref(pk)))
    return pk.as_dict()


def version() -> str:
    buf = C.create_string_buffer(256)
    lib.p2z_version(buf, 256)
    return buf.value.decode()


# ---------------------------------------------------------------------------
# AOSOA helpers
# ---------------------------------------------------------------------------

def trk_words(bsize: int) -> int:
    return TRK_WORDS * bsize


def hit_words(bsize: int) -> int:
    return HIT_WORDS * bsize


def empty_tracks(nbatches: int, bsize: int) -> np.ndarray:
    """float32 array of nbatches MPTRK batches (charge words hold int32 bits)."""
    return np.zeros((nbatches, TRK_WORDS, bsize), dtype=np.float32)


def empty_hits(nbatches: int, nlayer: int, bsize: int) -> np.ndarray:
    return np.zeros((nbatches, nlayer, HIT_WORDS, bsize), dtype=np.float32)


def tracks_to_aos(trk: np.ndarray) -> dict:
    """(nbatches, 28, B) AOSOA -> per-track arrays in slot order: par (n,6), cov (n,21), q (n,)."""
    nb, w, B = trk.shape
    assert w == TRK_WORDS
    t = np.ascontiguousarray(trk.transpose(0, 2, 1)).reshape(nb * B, TRK_WORDS)
    return {"par": t[:, :6].copy(), "cov": t[:, 6:27].copy(), "q": t[:, 27].copy().view(np.int32)}


def tracks_to_soa(trk: np.ndarray) -> np.ndarray:
    """(nbatches, 28, B) AOSOA -> (28, nslots) SoA (P2Z_LAYOUT_SOA), same slot order."""
    nb, w, B = trk.shape
    return np.ascontiguousarray(trk.transpose(1, 0, 2)).reshape(w, nb * B)


def hits_to_soa(hits: np.ndarray) -> np.ndarray:
    """(nbatches, nlayer, 9, B) AOSOA -> (nlayer, 9, nslots) SoA."""
    nb, nl, w, B = hits.shape
    return np.ascontiguousarray(hits.transpose(1, 2, 0, 3)).reshape(nl, w, nb * B)


def tracks_from_soa(trk: np.ndarray, bsize: int) -> np.ndarray:
    """(28, nslots) SoA -> (nslots/bsize, 28, bsize) AOSOA."""
    w, ns = trk.shape
    return np.ascontiguousarray(trk.reshape(w, ns // bsize, bsize).transpose(1, 0, 2))


def hits_from_soa(hits: np.ndarray, bsize: int) -> np.ndarray:
    """(nlayer, 9, nslots) SoA -> (nslots/bsize, nlayer, 9, bsize) AOSOA."""
    nl, w, ns = hits.shape
    return np.ascontiguousarray(hits.reshape(nl, w, ns // bsize, bsize).transpose(2, 0, 1, 3))


def hits_to_aos(hits: np.ndarray) -> dict:
    """(nbatches, nlayer, 9, B) -> pos (nslots, nlayer, 3), cov (nslots, nlayer, 6)."""
    nb, nl, w, B = hits.shape
    h = np.ascontiguousarray(hits.transpose(0, 3, 1, 2)).reshape(nb * B, nl, HIT_WORDS)
    return {"pos": h[:, :, :3].copy(), "cov": h[:, :, 3:].copy()}


def make_config(bsize=32, nevts=1, ntrks=None, nlayer=20, niter=1, kfact=0.0, update=UPDATE_V2,
                schedule=SCHED_AUTO, block_threads=0, flags=0, event_ntrks=None, layout=LAYOUT_AOSOA,
                threads_per_track=0):
    cfg = Config()
    cfg.abi_version = ABI_VERSION
    cfg.bsize = bsize
    cfg.nevts = nevts
    cfg.ntrks = ntrks if ntrks is not None else bsize
    cfg.nlayer = nlayer
    cfg.niter = niter
    cfg.kfact = kfact
    cfg.update = UPDATE_NAMES.get(update, update) if isinstance(update, str) else update
    cfg.schedule = SCHED_NAMES.get(schedule, schedule) if isinstance(schedule, str) else schedule
    cfg.block_threads = block_threads
    cfg.flags = flags
    cfg.layout = LAYOUT_NAMES.get(layout, layout) if isinstance(layout, str) else layout
    cfg.threads_per_track = threads_per_track
    if event_ntrks is not None:
        arr = np.ascontiguousarray(event_ntrks, dtype=np.int64)
        cfg._event_ntrks_keep = arr  # keep alive with the struct
        cfg.event_ntrks = arr.ctypes.data_as(C.POINTER(C.c_int64))
    return cfg


def num_batches(cfg: Config) -> int:
    n = lib.p2z_num_batches(C.byref(cfg))
    if n < 0:
        _check(BAD_ARG, None)
    return n


# cudaStreamLegacy: the legacy default stream, which the C API takes only as
# this explicit handle (a NULL stream means the context's own stream).
CUDA_STREAM_LEGACY = 0x1


def _torch_cuda(arrays):
    """The first torch CUDA tensor among arrays, or None."""
    for a in arrays:
        if a is not None and type(a).__module__.startswith("torch") and getattr(a, "is_cuda", False):
            return a
    return None


def _stream(stream, *arrays):
    """The stream handle a device call runs on.  An explicit stream (a handle
    or an object with .cuda_stream) is used as given.  Without one, a call on
    torch CUDA tensors runs on torch's current stream of their device: the
    library's kernels then follow the torch work that wrote those tensors, and
    no pending torch work can still be reading memory that torch's allocator
    has handed out again as one of them (the library's own stream is not
    ordered with torch's).  Otherwise None: the context's stream."""
    if stream is not None:
        h = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        return h if h != 0 else CUDA_STREAM_LEGACY
    t = _torch_cuda(arrays)
    if t is None:
        return None
    import torch
    h = torch.cuda.current_stream(t.device).cuda_stream
    return h if h != 0 else CUDA_STREAM_LEGACY


def _wait_for_torch(*arrays):
    """Before a call that runs on the context's stream only: wait for torch's
    current stream when torch CUDA tensors are among the arguments (the same
    ordering _stream gives the calls that take a stream)."""
    t = _torch_cuda(arrays)
    if t is not None:
        import torch
        torch.cuda.current_stream(t.device).synchronize()


def _ptr(a) -> int | None:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"]
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return int(a)


# ---------------------------------------------------------------------------
# Inputs and validation (host)
# ---------------------------------------------------------------------------

def make_atrk(par, cov, q) -> Atrk:
    t = Atrk()
    t.par[:] = [float(v) for v in par]
    t.cov[:] = [float(v) for v in cov]
    t.q = int(q)
    return t


def make_ahits(hits) -> C.Array:
    arr = (Ahit * len(hits))()
    for i, (pos, cov) in enumerate(hits):
        arr[i].pos[:] = [float(v) for v in pos]
        arr[i].cov[:] = [float(v) for v in cov]
    return arr


def prepare(seed: Atrk, hit_seeds, bsize, nevts, ntrks, nlayer, smear=1e-7, cov_scale=100.0):
    """The reference's srand(1) + prepareTracks + prepareHits (AOSOA numpy arrays)."""
    nb = nevts * (ntrks // bsize)
    trk = empty_tracks(nb, bsize)
    hit = empty_hits(nb, nlayer, bsize)
    _check(lib.p2z_prepare(C.byref(seed), hit_seeds, len(hit_seeds), bsize, nevts, ntrks, nlayer, smear, cov_scale,
                           _ptr(trk), _ptr(hit)))
    return trk, hit


def physics_params(**kw) -> PhysicsParams:
    p = PhysicsParams()
    lib.p2z_physics_defaults(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def generate_physics(cfg: Config, params: PhysicsParams | None = None, with_mask=False, out=None):
    """Physics workload into (trk, hits[, mask]) numpy arrays (or into `out`)."""
    params = params or physics_params()
    nb = num_batches(cfg)
    if out is None:
        trk = empty_tracks(nb, cfg.bsize)
        hit = empty_hits(nb, cfg.nlayer, cfg.bsize)
        mask = np.zeros(nb * cfg.bsize, dtype=np.uint32) if with_mask else None
    else:
        trk, hit, mask = out
    _check(lib.p2z_generate_physics(C.byref(params), C.byref(cfg), _ptr(trk), _ptr(hit), _ptr(mask)))
    return (trk, hit, mask) if with_mask else (trk, hit)


def mask_layers(mask: np.ndarray, nlayer, min_hits=5, max_hits=20, drop_prob=0.1, seed=7):
    _check(lib.p2z_mask_layers(_ptr(mask), mask.size, nlayer, min_hits, max_hits, drop_prob, seed))
    return mask


def validate(trk_out: np.ndarray, bsize, nevts, ntrks, hit_last) -> dict:
    v = Validation()
    hl = (C.c_float * 3)(*[float(x) for x in hit_last])
    _check(lib.p2z_validate(_ptr(trk_out), bsize, nevts, ntrks, hl, C.byref(v)))
    return v


def validate_sharded(trk_out: np.ndarray, bsize, nevts, ntrks, hit_last, allreduce=None) -> Validation:
    """Validation block of several event shards (one per process).  `allreduce`
    sums a float64 vector over all shards in place (e.g. a torch.distributed
    all-reduce); None means a single shard."""
    hl = (C.c_float * 3)(*[float(x) for x in hit_last])
    p1 = ValidationPartial()
    _check(lib.p2z_validate_partial(_ptr(trk_out), bsize, nevts, ntrks, hl, None, C.byref(p1)))
    if allreduce is not None:
        a = p1.to_array()
        allreduce(a)
        p1 = ValidationPartial.from_array(a)
    means = (C.c_double * 6)()
    lib.p2z_validate_means(C.byref(p1), means)
    p2 = ValidationPartial()
    _check(lib.p2z_validate_partial(_ptr(trk_out), bsize, nevts, ntrks, hl, means, C.byref(p2)))
    if allreduce is not None:
        a = p2.to_array()
        allreduce(a)
        p2 = ValidationPartial.from_array(a)
    v = Validation()
    _check(lib.p2z_validate_combine(C.byref(p1), C.byref(p2), C.byref(v)))
    return v


def shard_events(event_ntrks, world: int) -> list[tuple[int, int]]:
    """Contiguous event ranges [e0, e1) per rank with near-equal track counts
    (uniform events split evenly by count)."""
    counts = np.asarray(event_ntrks, dtype=np.int64)
    total = int(counts.sum())
    cum = np.concatenate([[0], np.cumsum(counts)])
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        e = int(np.searchsorted(cum, target, side="left"))
        e = max(bounds[-1], min(len(counts), e))
        if e > 0 and abs(cum[e - 1] - target) < abs(cum[e] - target) and e - 1 >= bounds[-1]:
            e -= 1
        bounds.append(e)
    bounds.append(len(counts))
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


def dump_tracks(trk_in, trk_out, bsize, nevts, ntrks, hit_last, directory=None):
    """The reference's DUMP_OUTPUT files (output_/input_ x, y, z .txt)."""
    h = (C.c_float * 3)(*hit_last)
    d = None if directory is None else str(directory).encode()
    _check(lib.p2z_dump_tracks(_ptr(trk_in), _ptr(trk_out), bsize, nevts, ntrks, h, d))


def print_validation(v: Validation):
    lib.p2z_print_validation(C.byref(v))


# ---------------------------------------------------------------------------
# Context
# ---------------------------------------------------------------------------

class Context:
    """Owns a p2z_context (device buffers, streams, graph cache) on one GPU."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(lib.p2z_create(device, C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            lib.p2z_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, cfg: Config, trk_in, hits, trk_out, hit_mask=None) -> Stats:
        """Host-memory pass (copies in, kernels, copies out)."""
        st = Stats()
        _check(lib.p2z_run(self.h, C.byref(cfg), _ptr(trk_in), _ptr(hits), _ptr(hit_mask), _ptr(trk_out),
                           C.byref(st)), self.h)
        return st

    def run_device(self, cfg: Config, d_trk_in, d_hits, d_trk_out, d_mask=None, stream=None, stats=True):
        """Device-memory pass; pointers are ints or objects with data_ptr()."""
        st = Stats() if stats else None
        stream = _stream(stream, d_trk_in, d_hits, d_mask, d_trk_out)
        _check(lib.p2z_run_device(self.h, C.byref(cfg), _ptr(d_trk_in), _ptr(d_hits), _ptr(d_mask),
                                  _ptr(d_trk_out), stream, C.byref(st) if st is not None else None), self.h)
        return st

    def step_device(self, bsize, nbatches, d_trk, d_hits, nlayer, layer, what=3, update=UPDATE_V2, kfact=0.0):
        _wait_for_torch(d_trk, d_hits)
        _check(lib.p2z_step_device(self.h, bsize, nbatches, _ptr(d_trk), _ptr(d_hits), nlayer, layer, what, update,
                                   kfact), self.h)

    def prepare_device(self, seed: Atrk, hit_seeds, bsize, nevts, ntrks, nlayer, d_trk, d_hits, smear=1e-7,
                       cov_scale=100.0, stream=None):
        """p2z_prepare on the device (p2z_prepare_device), into device buffers."""
        stream = _stream(stream, d_trk, d_hits)
        _check(lib.p2z_prepare_device(self.h, C.byref(seed), hit_seeds, len(hit_seeds), bsize, nevts, ntrks, nlayer,
                                      smear, cov_scale, _ptr(d_trk), _ptr(d_hits), stream), self.h)

    def generate_physics_device(self, cfg: Config, d_trk, d_hits, d_mask=None, params=None, stream=None):
        """The physics sample generated on the device (p2z_generate_physics_device)."""
        params = params or physics_params()
        stream = _stream(stream, d_trk, d_hits, d_mask)
        _check(lib.p2z_generate_physics_device(self.h, C.byref(params), C.byref(cfg), _ptr(d_trk), _ptr(d_hits),
                                               _ptr(d_mask), stream), self.h)

    def mask_layers_device(self, d_mask, nslots, nlayer, min_hits=5, max_hits=20, drop_prob=0.1, seed=7,
                           stream=None):
        stream = _stream(stream, d_mask)
        _check(lib.p2z_mask_layers_device(self.h, _ptr(d_mask), nslots, nlayer, min_hits, max_hits, drop_prob,
                                          seed, stream), self.h)

    def validate_device(self, d_trk_out, bsize, nevts, ntrks, hit_last, stream=None) -> dict:
        """The validation block reduced on the GPU (p2z_validate_device)."""
        h = (C.c_float * 3)(*hit_last)
        v = Validation()
        stream = _stream(stream, d_trk_out)
        _check(lib.p2z_validate_device(self.h, _ptr(d_trk_out), bsize, nevts, ntrks, h, C.byref(v), stream), self.h)
        return v

    def validate_partial_device(self, d_trk_out, bsize, nevts, ntrks, hit_last, means=None, stream=None):
        h = (C.c_float * 3)(*hit_last)
        m = None if means is None else (C.c_double * 6)(*means)
        acc = ValidationPartial()
        stream = _stream(stream, d_trk_out)
        _check(lib.p2z_validate_partial_device(self.h, _ptr(d_trk_out), bsize, nevts, ntrks, h, m, C.byref(acc),
                                               stream), self.h)
        return acc

    def relayout_device(self, cfg_from: Config, cfg_to: Config, d_trk_in, d_hits_in, d_trk_out, d_hits_out,
                        d_mask_in=None, d_mask_out=None, stream=None):
        """Convert device arrays between bsizes / AOSOA / SoA (p2z_relayout_device)."""
        stream = _stream(stream, d_trk_in, d_hits_in, d_mask_in, d_trk_out, d_hits_out, d_mask_out)
        _check(lib.p2z_relayout_device(self.h, C.byref(cfg_from), C.byref(cfg_to), _ptr(d_trk_in), _ptr(d_hits_in),
                                       _ptr(d_mask_in), _ptr(d_trk_out), _ptr(d_hits_out), _ptr(d_mask_out),
                                       stream), self.h)

    def pack_by_hits_device(self, cfg: Config, d_trk_in, d_hits_in, d_trk_out, d_hits_out, d_perm,
                            d_mask_in=None, d_mask_out=None, stream=None):
        """Copy of the arrays with every event's tracks in order of decreasing hit
        count, and in d_perm (2 x nslots int64) the input slot of every packed slot followed by
        the inverse (p2z_pack_by_hits_device)."""
        stream = _stream(stream, d_trk_in, d_hits_in, d_mask_in, d_trk_out, d_hits_out, d_mask_out, d_perm)
        _check(lib.p2z_pack_by_hits_device(self.h, C.byref(cfg), _ptr(d_trk_in), _ptr(d_hits_in), _ptr(d_mask_in),
                                           _ptr(d_trk_out), _ptr(d_hits_out), _ptr(d_mask_out), _ptr(d_perm),
                                           stream), self.h)

    def unpack_tracks_device(self, cfg: Config, d_perm, d_trk_packed, d_trk_out, stream=None):
        """A packed run's output back in the caller's slot order (p2z_unpack_tracks_device)."""
        stream = _stream(stream, d_perm, d_trk_packed, d_trk_out)
        _check(lib.p2z_unpack_tracks_device(self.h, C.byref(cfg), _ptr(d_perm), _ptr(d_trk_packed), _ptr(d_trk_out),
                                            stream), self.h)

    def autotune(self, cfg: Config, d_trk_in, d_hits, d_mask=None, reps=3, max_entries=1024):
        """Measure every bsize x layout x schedule x block size (p2z_autotune).
        Returns (best, entries) as dicts, entries sorted by time."""
        rows = (TuneEntry * max_entries)()
        n = C.c_int(0)
        best = TuneEntry()
        _wait_for_torch(d_trk_in, d_hits, d_mask)
        _check(lib.p2z_autotune(self.h, C.byref(cfg), _ptr(d_trk_in), _ptr(d_hits), _ptr(d_mask), reps, rows,
                                max_entries, C.byref(n), C.byref(best)), self.h)
        entries = sorted((rows[i].as_dict() for i in range(min(n.value, max_entries))), key=lambda d: d["ms"])
        return best.as_dict(), entries


class Server:
    """Continuous-batching server (p2z_server_*).  Host arrays handed to
    submit() are kept referenced until their request is reported."""

    def __init__(self, device=0, bsize=32, nlayer=20, update=UPDATE_V2, flags=0, budget_bytes=1 << 30,
                 max_inflight=2, block_threads=0, kfact=0.0):
        cfg = ServerConfig()
        cfg.abi_version = ABI_VERSION
        cfg.bsize = bsize
        cfg.nlayer = nlayer
        cfg.update = UPDATE_NAMES.get(update, update) if isinstance(update, str) else update
        cfg.flags = flags
        cfg.kfact = kfact
        cfg.device_budget_bytes = int(budget_bytes)
        cfg.max_inflight = max_inflight
        cfg.block_threads = block_threads
        h = C.c_void_p()
        _check(lib.p2z_server_create(device, C.byref(cfg), C.byref(h)))
        self.h = h
        self.bsize = bsize
        self._keep = {}

    def submit(self, trk, hits, mask, ntrks, out) -> int:
        rid = C.c_int64()
        _check(lib.p2z_server_submit(self.h, _ptr(trk), _ptr(hits), _ptr(mask), int(ntrks), _ptr(out), C.byref(rid)))
        self._keep[rid.value] = (trk, hits, mask, out)
        return rid.value

    def poll(self, rid):
        info = RequestInfo()
        st = lib.p2z_server_poll(self.h, rid, C.byref(info))
        if st == NOT_READY:
            return None
        _check(st)
        self._keep.pop(rid, None)
        return info

    def wait(self, rid, timeout=600.0) -> RequestInfo:
        info = RequestInfo()
        _check(lib.p2z_server_wait(self.h, rid, timeout, C.byref(info)))
        self._keep.pop(rid, None)
        return info

    def now(self) -> float:
        return lib.p2z_server_now(self.h)

    def replay(self, events, arrivals):
        """events: list of (trk, hits, mask, ntrks, out); arrivals: seconds from now."""
        n = len(events)
        P = C.c_void_p * n
        trk = P(*[_ptr(e[0]) for e in events])
        hit = P(*[_ptr(e[1]) for e in events])
        msk = P(*[_ptr(e[2]) for e in events])
        ntr = (C.c_int64 * n)(*[int(e[3]) for e in events])
        out = P(*[_ptr(e[4]) for e in events])
        arr = (C.c_double * n)(*[float(a) for a in arrivals])
        infos = (RequestInfo * n)()
        _check(lib.p2z_server_replay(self.h, n, trk, hit, msk, ntr, out, arr, infos))
        return list(infos)

    def close(self):
        if self.h:
            lib.p2z_server_destroy(self.h)
            self.h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class PinnedArray:
    """numpy view of page-locked host memory from p2z_host_alloc."""

    def __init__(self, shape, dtype=np.float32):
        n = int(np.prod(shape)) * np.dtype(dtype).itemsize
        p = C.c_void_p()
        _check(lib.p2z_host_alloc(C.byref(p), n))
        self._p = p
        buf = (C.c_char * n).from_address(p.value)
        self.array = np.frombuffer(buf, dtype=dtype).reshape(shape)

    def free(self):
        if self._p:
            self.array = None
            lib.p2z_host_free(self._p)
            self._p = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
