"""The C++ code in INTEGRATION.md compiles where a maintainer would paste it:
the C ABI snippets (replacing the OpenMP build's timed loop, the CUDA_v4
build's per-stream launches, and packing by hit count) inside functions of a
translation unit that defines the reference's size macros before the header,
as src/propagate-toz-test_OMP.cpp does; the typed example as a program of its
own.  Syntax only: nothing runs.  CPU."""
import re
import shutil
import subprocess

import pytest

from conftest import ROOT

GUIDE = ROOT / "INTEGRATION.md"
CUDA_INCLUDE = "/usr/local/cuda/include"

PRELUDE = """#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <cuda_runtime.h>
#define bsize 32
#define nevts 100
#define ntrks 9600
#define nb (ntrks / bsize)
#define nlayer 20
#define NITER 5
#define smear 0.0000001
#define nthreads 64
#define N bsize
#define num_streams 10
struct MPTRK { float par[6 * bsize]; float cov[21 * bsize]; int q[bsize]; };
struct MPHIT { float pos[3 * bsize]; float cov[6 * bsize]; };
"""


def _blocks():
    return re.findall(r"```cpp\n(.*?)```", GUIDE.read_text(), re.S)


def _compile(tmp_path, name, source):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    src = tmp_path / name
    src.write_text(source)
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", f"-I{ROOT / 'include'}", f"-I{CUDA_INCLUDE}",
                        str(src)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr + "\n" + source


def test_guide_has_the_snippets():
    b = _blocks()
    assert len(b) == 4
    assert "p2z_run(" in b[1] and "p2z_run_device(" in b[2] and "p2z_pack_by_hits_device(" in b[3]


def test_c_abi_snippets_compile_in_the_reference_setting(tmp_path):
    typed, timed_loop, streams, packing = _blocks()
    include = [l for l in timed_loop.splitlines() if l.startswith("#include")]
    body = "\n".join(l for l in timed_loop.splitlines() if not l.startswith("#include"))
    assert include == ['#include "p2z.h"   // with the other includes, or anywhere after the size macros: it '
                       'sets them aside']
    src = (PRELUDE + include[0] + "\n"
           "void replace_timed_loop(MPTRK *trk, MPHIT *hit, MPTRK *outtrk) {\n" + body + "\n}\n"
           "void replace_stream_launches(p2z_context *ctx, MPTRK *trk_dev, MPHIT *hit_dev, MPTRK *outtrk_dev,\n"
           "                             cudaStream_t *streams, int stream_chunk) {\n" + streams + "\n}\n"
           "void packed_passes(p2z_context *ctx, p2z_config cfg, const void *d_trk, const void *d_hits,\n"
           "                   const uint32_t *d_mask, void *d_trk_p, void *d_hits_p, uint32_t *d_mask_p,\n"
           "                   int64_t *d_perm, void *d_out_p, void *d_out, void *stream, int npasses) {\n"
           + packing + "\n}\n")
    _compile(tmp_path, "c_abi_snippets.cpp", src)


def test_typed_example_compiles(tmp_path):
    typed = _blocks()[0]
    # the example leaves the seed values to the reader
    src = typed.replace("= /* the seed track */;", "{};").replace("= /* one seed hit per layer */;", "(nlayer);")
    assert src != typed
    _compile(tmp_path, "typed_example.cpp", src)
