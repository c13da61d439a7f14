"""The C ABI without a GPU: the library loads, exports every entry point that
include/flip2_b200.h declares, the Python mirror binds them, and calls that
need a device fail with a status instead of exiting the process."""
import ctypes as C
import os
import re
import subprocess

import pytest

import flip2_b200 as F

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    syms = F.exported_symbols()
    assert len(syms) >= 40
    out = subprocess.run(["nm", "-D", "--defined-only", F.LIB_PATH], capture_output=True, text=True, check=True).stdout
    defined = set(re.findall(r" T (\w+)$", out, flags=re.M))
    missing = [s for s in syms if s not in defined]
    assert not missing, missing


def test_library_loads_and_binds():
    L = F.lib()
    assert b"sm_100a" in L.flip_version()
    assert L.flip_status_string(5) == b"call out of order"
    for s in F.exported_symbols():
        assert hasattr(L, s)


def test_sm100a_build_flags():
    """Every object of the library is compiled for sm_100a and nothing else."""
    from flip2_b200 import build as B
    assert B.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert "-gencode" not in " ".join(B.NVCC_FLAGS).replace(" ".join(B.ARCH), "")


@pytest.mark.gpu
def test_sm100a_code_loaded():
    """The runtime loads sm_100 device code for the library's kernels
    (cudaFuncAttributes::binaryVersion through the C ABI)."""
    L = F.lib()
    v = C.c_int(0)
    assert L.flip_binary_version(C.byref(v)) == 0
    assert v.value == 100, v.value


def test_scratch_size_queries():
    L = F.lib()
    assert L.flip_sort_pairs_scratch_bytes(1 << 26) > 8 * (1 << 26)
    assert L.flip_inclusive_scan_scratch_bytes(4096) >= 8
    assert L.flip_segment_heads_scratch_bytes(10) >= 8


def test_bad_arguments_return_status():
    L = F.lib()
    assert L.flip_sort_pairs(None, None, None, None, 10, 32, None, 0, None) == 1
    assert L.flip_sort_pairs(None, None, None, None, 0, 32, None, 0, None) == 0
    h = C.c_void_p()
    assert L.flip_create(0, None, None, C.byref(h)) == 1


def test_create_without_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    L = F.lib()
    h = C.c_void_p()
    rc = L.flip_create(1000, None, None, C.byref(h))
    assert rc == 7 and not h.value
    assert b"device" in L.flip_last_error(None)


def test_params_layout_matches_header():
    hdr = open(os.path.join(ROOT, "include", "flip2_b200.h")).read()
    body = hdr[hdr.index("typedef struct {\n    int32_t mode;"):]
    body = body[:body.index("} flip_params;")]
    fields = re.findall(r"\b(?:int32_t|float|double)\s+(\w+)(?:\[(\d+)\])?;", body)
    names = [f[0] for f in fields]
    assert names == [f[0] for f in F.Params._fields_]
    # offsets and size as the C compiler lays the struct out
    import shutil
    import tempfile
    cc = shutil.which("x86_64-linux-gnu-gcc-13") or shutil.which("gcc")
    if cc is None:
        pytest.skip("no C compiler")
    prog = '#include <stdio.h>\n#include <stddef.h>\n#include "flip2_b200.h"\nint main(void){' + "".join(
        'printf("%%zu ", offsetof(flip_params, %s));' % n for n in names) + 'printf("%zu", sizeof(flip_params));return 0;}'
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "p.c"), os.path.join(d, "p")
        open(src, "w").write(prog)
        subprocess.run([cc, "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        got = [int(v) for v in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()]
    assert got[:-1] == [getattr(F.Params, n).offset for n in names]
    assert got[-1] == C.sizeof(F.Params)
