"""The C-ABI library loads and exports every entry point of include/dnsbox.h,
and the ctypes mirrors of its structs have the C layout (no GPU needed)."""
import ctypes
import os
import re
import subprocess

import pytest

from dnsbox_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "dnsbox.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(dnsbox_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "dnsbox_rhs_nonlinear" in names and "dnsbox_step" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libdnsbox_gpu.so not built")
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers the whole header
    assert set(declared_functions()) <= set(_lib.SIGNATURES)


def test_library_host_only_calls():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libdnsbox_gpu.so not built")
    lib = _lib.load()
    assert lib.dnsbox_abi_version() == 1
    for n in (8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256, 512, 1024):
        assert lib.dnsbox_supported_size(n) == 1
    for n in (0, 10, 100, 2048):
        assert lib.dnsbox_supported_size(n) == 0
    p = _lib.Params()
    lib.dnsbox_default_params(ctypes.byref(p))
    assert (p.nx, p.nu, p.Pin, p.kCutOff, p.courant_max) == (128, 0.005, 0.1, 2.0, 0.2)
    # argument errors are reported without touching a GPU
    h = ctypes.c_void_p()
    p.nx = 100
    assert lib.dnsbox_create(ctypes.byref(p), ctypes.byref(h)) == -2
    assert b"unsupported grid" in lib.dnsbox_last_error()
    assert lib.dnsbox_create(None, ctypes.byref(h)) == -1
    assert lib.dnsbox_step(None, None, 1, None) == -1


def test_struct_layouts_match_c(tmp_path):
    prog = tmp_path / "sz.c"
    prog.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "dnsbox.h"\n'
                    'int main(){printf("%zu %zu %zu %zu\\n", sizeof(dnsbox_params), sizeof(dnsbox_diag),'
                    ' offsetof(dnsbox_params, nu), offsetof(dnsbox_diag, nonfinite)); return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(prog), "-o", str(exe)])
    out = subprocess.check_output([str(exe)]).decode().split()
    assert int(out[0]) == ctypes.sizeof(_lib.Params)
    assert int(out[1]) == ctypes.sizeof(_lib.Diag)
    assert int(out[2]) == _lib.Params.nu.offset
    assert int(out[3]) == _lib.Diag.nonfinite.offset


def test_torch_operator_library_registers():
    """torch.ops.dnsbox.* (csrc/torch_ops.cpp) loads without a GPU and declares
    the operators with their schemas."""
    from dnsbox_b200 import torch_ops
    if not os.path.exists(torch_ops.OUT):
        pytest.skip("libdnsbox_torch.so not built")
    ops = torch_ops.load()
    names = ["rhs_nonlinear", "rhs_nonlinear_vjp", "step_", "residual", "residual_grad", "c2r", "r2c"]
    for n in names:
        assert hasattr(ops, n)
    assert "Tensor(a!)" in str(ops.step_.default._schema)
