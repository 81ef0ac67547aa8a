"""PyTorch operator library ``torch.ops.dnsbox.*`` over the C ABI.

``csrc/torch_ops.cpp`` registers the operators with the dispatcher for CUDA
tensors (no CPU path); they run on torch's current stream and allocate through
the caching allocator.  ``build()`` compiles it in-tree next to
libdnsbox_gpu.so (``_lib/libdnsbox_torch.so``); ``load()`` registers it.  The
context argument is ``Box.handle``.  ``rhs_nonlinear`` gets an autograd rule
whose backward is the exact transpose ``rhs_nonlinear_vjp`` (the counterpart
of rhsAdj.f90's adjoint nonlinear term).
"""
from __future__ import annotations

import os
import subprocess

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc", "torch_ops.cpp")
OUT = os.path.join(HERE, "_lib", "libdnsbox_torch.so")
_loaded = False


def build(force: bool = False) -> str:
    """Compiles csrc/torch_ops.cpp against torch's headers and libraries."""
    from torch.utils.cpp_extension import include_paths, library_paths
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= os.path.getmtime(SRC):
        return OUT
    inc = include_paths(device_type="cuda")
    libs = library_paths(device_type="cuda")
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", f"-D_GLIBCXX_USE_CXX11_ABI={abi}",
           *[f"-I{p}" for p in inc], SRC, "-o", OUT,
           *[f"-L{p}" for p in libs], "-L" + os.path.join(HERE, "_lib"),
           "-Wl,--no-as-needed", "-ldnsbox_gpu", "-lc10", "-lc10_cuda", "-ltorch_cpu", "-ltorch_cuda", "-ltorch",
           "-lcudart", "-Wl,-rpath,$ORIGIN"]
    subprocess.check_call(cmd)
    return OUT


def load():
    """Registers torch.ops.dnsbox (raises if the library is not built)."""
    global _loaded
    if _loaded:
        return torch.ops.dnsbox
    if not os.path.exists(OUT):
        raise RuntimeError(f"{OUT} is not built (run __graft_entry__.build())")
    from . import _lib
    _lib.load()   # libdnsbox_gpu.so first (the operator library links against it)
    torch.ops.load_library(OUT)

    def _setup(ctx, inputs, output):
        ctx.h, ctx.uh = inputs[0], inputs[1]

    def _backward(ctx, grad):
        return None, torch.ops.dnsbox.rhs_nonlinear_vjp(ctx.h, ctx.uh, grad.contiguous())

    torch.library.register_autograd("dnsbox::rhs_nonlinear", _backward, setup_context=_setup)
    _loaded = True
    return torch.ops.dnsbox
