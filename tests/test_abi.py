"""The C-ABI library: it loads, exports every entry point include/huntian_b200.h declares
(and nothing else), and fails cleanly -- status code plus message, no crash -- when no GPU
is usable.  No compute calls; runs without a GPU."""
import ctypes as C
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "huntian_b200.h")


def _declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"HT_API\s+(?:int|const char\*)\s+(ht_\w+)\(", txt)))


def test_header_matches_binding_table(ht):
    assert _declared() == sorted(ht.SYMBOLS)


def test_library_exports_every_declared_symbol(ht):
    lib = ht._lib.load()
    for name in _declared():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", ht.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = sorted(ln.split()[-1] for ln in out.splitlines() if " T " in ln)
    assert exported == _declared()


def test_checked_library_exports_the_same_symbols(ht):
    """libhuntian_b200_checked.so (build.py --checked, -DHT_CHECKED) is the same C ABI:
    every declared entry point and nothing else."""
    path = os.path.join(os.path.dirname(ht.LIB_PATH), "libhuntian_b200_checked.so")
    if not os.path.exists(path):
        pytest.skip("checked build not present (python huntian.jl_b200/build.py --checked)")
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True,
                         text=True, check=True).stdout
    exported = sorted(ln.split()[-1] for ln in out.splitlines() if " T " in ln)
    assert exported == _declared()


def test_errors_are_status_codes(ht):
    lib = ht._lib.load()
    h = C.c_void_p()
    # argument checks come before any device call
    rc = lib.ht_ctx_create(0, 0, None, 2, 2, 2, 0, 1, 0, 1, 0, 1, -1.0, C.byref(h))
    assert rc == ht._lib.HT_ERR_INVALID
    assert b"nhunt" in lib.ht_last_error()
    rc = lib.ht_shell_analyse(None, None, 1.0, 0.0, 0, None, 0, 0, None, None)
    assert rc == ht._lib.HT_ERR_INVALID and lib.ht_last_error()


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES", None) is None and
                    os.path.exists("/dev/nvidia0"), reason="GPU present")
def test_no_gpu_gives_cuda_error(ht):
    import numpy as np
    lib = ht._lib.load()
    tab = np.zeros(8, np.float32)
    h = C.c_void_p()
    rc = lib.ht_ctx_create(0, 4, tab.ctypes.data, 2, 2, 2, 0, 1, 0, 1, 0, 1, -1.0, C.byref(h))
    assert rc == ht._lib.HT_ERR_CUDA and lib.ht_last_error()
