"""ctypes access to the CHECKERS -- test infrastructure, never product code.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
legs import this module.  It loads:

* ``liboracle.so`` -- this repository's C restatement of the reference's
  per-track arithmetic (p2z_oracle.c): FP32 in the reference's own semantics,
  and the FP64 host oracle.
* ``_ref/<isa>/libp2zref_*.so`` -- the reference benchmark's own OpenMP source
  (src/propagate-toz-test_OMP.cpp) compiled unchanged by oracle/Makefile.

``physics()`` generates the benchmark's physics sample from the restatement
in p2z_physics_oracle.c (part of liboracle.so), so that the benchmark's
reference arm builds its inputs without the product library.

Both are built by ``make -C oracle oracle ref`` (the ``ref`` target needs the
reference tree; its outputs travel with the repository snapshot).
"""
from __future__ import annotations

import ctypes as C
import pathlib

import numpy as np

ORACLE_DIR = pathlib.Path(__file__).resolve().parent
REF_DIR = ORACLE_DIR / "_ref"

UPDATE_V2 = 0
UPDATE_3X3_JOSEPH = 1


def host_isa() -> str:
    """'v4' when the host CPU has AVX-512 (F, BW, CD, DQ, VL), else 'v3'."""
    try:
        flags = set()
        for line in open("/proc/cpuinfo"):
            if line.startswith("flags"):
                flags = set(line.split(":", 1)[1].split())
                break
        if {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"} <= flags:
            return "v4"
    except OSError:
        pass
    return "v3"


_oracle = {}


def oracle_lib(cr_trig: bool = False):
    """cr_trig: the build whose sinf/cosf are correctly rounded (else the C library's)."""
    key = bool(cr_trig)
    if key not in _oracle:
        path = ORACLE_DIR / ("liboracle_crtrig.so" if key else "liboracle.so")
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (make -C oracle oracle)")
        lib = C.CDLL(str(path))
        lib.orc_default_kfact.restype = C.c_float
        lib.orc_run_f32.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_void_p,
                                    C.c_float]
        lib.orc_run_f32.restype = None
        lib.orc_step_f32.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_float]
        lib.orc_step_f32.restype = None
        lib.orc_run_f64.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_void_p,
                                    C.c_double, C.c_int]
        lib.orc_run_f64.restype = None
        _oracle[key] = lib
    return _oracle[key]


def _p(a):
    return None if a is None else a.ctypes.data


class PhysicsParams(C.Structure):
    """The physics sample's parameters (field order of the library's
    p2z_physics_params; defaults: the benchmark's physics workload)."""
    _fields_ = [("seed", C.c_uint64), ("pt_min", C.c_double), ("pt_max", C.c_double), ("eta_min", C.c_double),
                ("eta_max", C.c_double), ("sigma_vz", C.c_double), ("sig_xy", C.c_double), ("sig_z", C.c_double),
                ("rel_sig_ipt", C.c_double), ("sig_phi", C.c_double), ("sig_theta", C.c_double),
                ("rho_max", C.c_double), ("z_first", C.c_double), ("z_last", C.c_double),
                ("hit_sig_xy", C.c_double), ("hit_sig_z", C.c_double), ("kfact", C.c_float),
                ("nthreads", C.c_int32)]

    DEFAULTS = dict(seed=20240601, pt_min=0.5, pt_max=20.0, eta_min=1.6, eta_max=2.5, sigma_vz=5.0, sig_xy=0.01,
                    sig_z=0.05, rel_sig_ipt=0.01, sig_phi=1e-3, sig_theta=1e-3, rho_max=0.3, z_first=30.0,
                    z_last=270.0, hit_sig_xy=30e-4, hit_sig_z=1e-4, kfact=0.0, nthreads=0)

    def __init__(self, **kw):
        super().__init__(**{**self.DEFAULTS, **kw})


def physics(bsize: int, nevts: int, ntrks: int, nlayer: int = 20, **params):
    """The physics sample (uniform events) as (trk (nb,28,B), hits (nb,nl,9,B)) float32."""
    lib = oracle_lib()
    lib.oph_generate.argtypes = [C.c_void_p, C.c_int, C.c_int64, C.c_int64, C.c_int, C.c_void_p, C.c_void_p]
    lib.oph_generate.restype = C.c_int
    nb = nevts * ntrks // bsize
    trk = np.empty((nb, 28, bsize), dtype=np.float32)
    hit = np.empty((nb, nlayer, 9, bsize), dtype=np.float32)
    prm = PhysicsParams(**params)
    if lib.oph_generate(C.byref(prm), bsize, nevts, ntrks, nlayer, _p(trk), _p(hit)):
        raise ValueError("bad physics sample size")
    return trk, hit


def kfact_default() -> float:
    return float(oracle_lib().orc_default_kfact())


def run_f32(trk: np.ndarray, hits: np.ndarray, mask=None, kfact=None, cr_trig=False) -> np.ndarray:
    """Restatement, reference FP32 semantics.  trk (nb,28,B) float32, hits (nb,nl,9,B)."""
    nb, _, B = trk.shape
    nl = hits.shape[1]
    out = np.empty_like(trk)
    oracle_lib(cr_trig).orc_run_f32(_p(trk), _p(hits), _p(out), nb, B, nl, _p(mask),
                             kfact_default() if kfact is None else kfact)
    return out


def step_f32(batch: np.ndarray, hitbatch: np.ndarray, which: int, kfact=None):
    """In-place single step on one batch: which 0 = propagate, 1 = update_v2."""
    B = batch.shape[-1]
    oracle_lib().orc_step_f32(_p(batch), _p(hitbatch), B, which, kfact_default() if kfact is None else kfact)


def run_f64(trk: np.ndarray, hits: np.ndarray, mask=None, kfact=None, update=UPDATE_V2) -> np.ndarray:
    """FP64 host oracle; returns (nslots, 27) float64: 6 parameters, 21 covariance."""
    nb, _, B = trk.shape
    nl = hits.shape[1]
    out = np.empty((nb * B, 27), dtype=np.float64)
    oracle_lib().orc_run_f64(_p(trk), _p(hits), _p(out), nb, B, nl, _p(mask),
                             kfact_default() if kfact is None else kfact, update)
    return out


# ---------------------------------------------------------------------------
# The reference itself
# ---------------------------------------------------------------------------

class RefAtrk(C.Structure):
    _fields_ = [("par", C.c_float * 6), ("cov", C.c_float * 21), ("q", C.c_int)]


class RefAhit(C.Structure):
    _fields_ = [("pos", C.c_float * 3), ("cov", C.c_float * 6)]


_refs = {}


def ref_available(name: str = "b32") -> bool:
    return (REF_DIR / host_isa() / f"libp2zref_{name}.so").exists()


def ref_lib(name: str = "b32"):
    """The reference compiled unchanged; name: b8/b16/b32/b64 (2x128 prepare
    sizes), kat (100x9600, bsize 32), b32_nofma (-ffp-contract=off) or
    b32_nofma_crtrig (-ffp-contract=off, sinf/cosf bound to correctly rounded
    versions)."""
    key = (host_isa(), name)
    if key not in _refs:
        path = REF_DIR / key[0] / f"libp2zref_{name}.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (make -C oracle ref, needs the reference tree)")
        lib = C.CDLL(str(path))
        for fn in ("ref_bsize", "ref_nevts", "ref_ntrks", "ref_nlayer"):
            getattr(lib, fn).restype = C.c_int
        lib.ref_kfact.restype = C.c_float
        lib.ref_sizeof_mptrk.restype = C.c_size_t
        lib.ref_sizeof_mphit.restype = C.c_size_t
        lib.ref_kat_seed.argtypes = [C.POINTER(RefAtrk), C.POINTER(RefAhit)]
        lib.ref_prepare.argtypes = [C.POINTER(RefAtrk), C.POINTER(RefAhit), C.c_int, C.c_void_p, C.c_void_p]
        lib.ref_prepare.restype = C.c_int
        lib.ref_run.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_long, C.c_long, C.c_int, C.c_int]
        lib.ref_run.restype = None
        lib.ref_propagate_batch.argtypes = [C.c_void_p, C.c_void_p]
        lib.ref_update_v2_batch.argtypes = [C.c_void_p, C.c_void_p]
        lib.ref_main.restype = C.c_int
        _refs[key] = lib
    return _refs[key]


def ref_kat_seed():
    """The reference's known-answer seed: (par, cov, q), [(pos, cov)] * 26 in layer order."""
    lib = ref_lib("b32")
    t = RefAtrk()
    h = (RefAhit * 26)()
    lib.ref_kat_seed(C.byref(t), h)
    return (list(t.par), list(t.cov), t.q), [(list(x.pos), list(x.cov)) for x in h]


def ref_prepare(name: str, seed, hits):
    """srand(1) + the reference's prepareTracks/prepareHits at that library's sizes."""
    lib = ref_lib(name)
    B, nev, ntrk, nl = lib.ref_bsize(), lib.ref_nevts(), lib.ref_ntrks(), lib.ref_nlayer()
    nb = nev * (ntrk // B)
    t = RefAtrk()
    t.par[:] = seed[0]
    t.cov[:] = seed[1]
    t.q = seed[2]
    h = (RefAhit * len(hits))()
    for i, (p, c) in enumerate(hits):
        h[i].pos[:] = p
        h[i].cov[:] = c
    trk = np.zeros((nb, 28, B), dtype=np.float32)
    hit = np.zeros((nb, nl, 9, B), dtype=np.float32)
    rc = lib.ref_prepare(C.byref(t), h, len(hits), _p(trk), _p(hit))
    if rc:
        raise ValueError("reference prepare failed (too few hits)")
    return trk, hit


def ref_run(trk: np.ndarray, hits: np.ndarray, nev: int | None = None, nthreads: int = 0, name=None) -> np.ndarray:
    """The reference's hot loop (propagateToZ + KalmanUpdate_v2 per layer)."""
    nb, _, B = trk.shape
    nl = hits.shape[1]
    lib = ref_lib(name or f"b{B}")
    assert lib.ref_bsize() == B
    out = np.empty_like(trk)
    if nev is None:
        nev = 1
    assert nb % nev == 0
    lib.ref_run(_p(trk), _p(hits), _p(out), nev, nb // nev, nl, nthreads)
    return out
