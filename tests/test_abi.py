"""The C-ABI library loads and exports every symbol include/chanrhs.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

from compchan3dmpi_b200 import _lib

ROOT = Path(__file__).resolve().parent.parent


def header_functions():
    src = (ROOT / "include" / "chanrhs.h").read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(chan_[a-z_0-9]+)\s*\(", src)))


@pytest.fixture(scope="module")
def built():
    from compchan3dmpi_b200.build import build
    return build()


def test_header_declares_expected_api():
    names = header_functions()
    for need in ("chan_init", "chan_upload", "chan_stage", "chan_step", "chan_stats", "chan_download",
                 "chan_set_forcing", "chan_status", "chan_free"):
        assert need in names


def test_library_exports_every_declared_symbol(built):
    L = ctypes.CDLL(str(built))
    for name in header_functions():
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(built)], capture_output=True, text=True).stdout
    for name in header_functions():
        assert re.search(rf"\bT {name}\b", out), name


def test_python_binding_covers_header():
    bound = {n for n, _, _ in _lib.SIGNATURES}
    assert bound == set(header_functions())


def test_struct_layout_matches_header():
    # offsets of chan_params as a C compiler lays it out
    code = r'''
#include <stdio.h>
#include <stddef.h>
#include "chanrhs.h"
int main(void){printf("%zu %zu %zu %zu %zu %zu\n", sizeof(chan_params), offsetof(chan_params, Re),
 offsetof(chan_params, Pe), offsetof(chan_params, Lx), offsetof(chan_params, Tw), offsetof(chan_params, flags));return 0;}
'''
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        c = Path(d) / "t.c"
        c.write_text(code)
        exe = Path(d) / "t"
        subprocess.run(["gcc", "-I", str(ROOT / "include"), "-o", str(exe), str(c)], check=True)
        vals = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    C = _lib.ChanParamsC
    assert vals == [ctypes.sizeof(C), C.Re.offset, C.Pe.offset, C.Lx.offset, C.Tw.offset, C.flags.offset]


def test_version_without_gpu(built):
    L = _lib.load()
    assert b"sm_100a" in L.chan_version()


def test_init_rejects_bad_arguments_without_gpu(built):
    import numpy as np
    L = _lib.load()
    p = _lib.ChanParamsC()
    p.nP[:] = [4, 8, 9]
    x = np.linspace(0, 2, 9)
    h = ctypes.c_void_p()
    assert L.chan_init(ctypes.byref(p), _lib.dptr(x), _lib.dptr(x), _lib.dptr(x), ctypes.byref(h)) == -1
    assert b"nP" in L.chan_last_error(None)
    assert L.chan_init(None, None, None, None, ctypes.byref(h)) == -1
