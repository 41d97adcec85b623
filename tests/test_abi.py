"""The C ABI on the CPU: the library loads without a GPU, exports every function include/rbmd_gpu.h
declares (read from the header itself), and its host-only entry points work."""
import ctypes as C
import os
import re
import subprocess

import pytest

import rbmd_b200
from rbmd_b200 import _abi as A

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rbmd_gpu.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rbmd_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_python_table():
    assert header_functions() == sorted(A.HEADER_FUNCTIONS)


def test_library_exports_every_header_function():
    L = rbmd_b200.lib()
    missing = [f for f in header_functions() if not hasattr(L, f)]
    assert not missing
    out = subprocess.run(["nm", "-D", "--defined-only", rbmd_b200.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (rbmd_[a-z0-9_]+)$", out, flags=re.M))
    assert set(header_functions()) <= exported


def test_header_compiles_as_c():
    """The boundary is plain C: the header must compile with a C compiler, no C++ types."""
    src = '#include "rbmd_gpu.h"\nint main(void) { rbmd_params p; rbmd_params_default(&p); return p.neighbor; }\n'
    r = subprocess.run(["gcc", "-std=c99", "-fsyntax-only", "-I", os.path.dirname(HEADER), "-x", "c", "-"],
                       input=src, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_host_only_entry_points():
    L = rbmd_b200.lib()
    assert L.rbmd_abi_version() == A.RBMD_ABI_VERSION == 6
    p = A.Params()
    L.rbmd_params_default(C.byref(p))
    assert p.neighbor == A.NEIGH_RBL and p.precision == A.PREC_FP64 and p.fix_shake == A.SHAKE_NULL
    # null arguments are status codes, never crashes
    assert L.rbmd_ctx_destroy(None) != 0
    assert L.rbmd_system_bytes(None, None, None) == A.ERR_ARG
    assert L.rbmd_eam_read_funcfl(b"/nonexistent/file.eam", C.byref(A.EamFile()), None, None, None) == A.ERR_IO


def test_struct_sizes_match_header(tmp_path):
    """ctypes mirrors of the ABI structs have the C layout (sizes from a C compile of the header)."""
    src = ('#include <stdio.h>\n#include "rbmd_gpu.h"\nint main(void) { printf("%zu %zu %zu %zu %zu %zu %zu %zu\\n", '
           'sizeof(rbmd_params), sizeof(rbmd_system_desc), sizeof(rbmd_thermo), sizeof(rbmd_serve_cfg), '
           'sizeof(rbmd_request_stats), sizeof(rbmd_device_cfg), sizeof(rbmd_tune_result), sizeof(rbmd_eam_setfl)); return 0; }\n')
    exe = str(tmp_path / "abi_sizes")
    r = subprocess.run(["gcc", "-I", os.path.dirname(HEADER), "-x", "c", "-", "-o", exe], input=src,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    sizes = list(map(int, subprocess.run([exe], capture_output=True, text=True).stdout.split()))
    assert sizes == [C.sizeof(A.Params), C.sizeof(A.SystemDesc), C.sizeof(A.Thermo), C.sizeof(A.ServeCfg),
                     C.sizeof(A.RequestStats), C.sizeof(A.DeviceCfg), C.sizeof(A.TuneResult), C.sizeof(A.EamSetfl)]
