"""dnsbox_c2r_noalloc, the allocation-free 3D C2R, against dnsbox_c2r.

The entry point serves callers that cannot allocate device memory (their
memory belongs to a pool they must not bypass, or allocating is not allowed
where they run); it keeps its intermediate fields in a static device array.
This file is collected last so that a run stopping at the first failure has
run every other test first; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float((a - b).norm() / b.norm())


@pytest.mark.parametrize("prec,shape,tol", [("fp64", (64, 64, 64), 1e-13),   # transform tolerances
                                            ("fp32", (96, 48, 64), 2e-6)])
def test_c2r_noalloc_matches_c2r_twice(prec, shape, tol):
    from dnsbox_b200 import _lib
    from dnsbox_b200.ops import PRECISION, Box
    nx, ny, nz = shape
    lib = _lib.load()
    box = Box(nx=nx, ny=ny, nz=nz, precision=prec)
    rng = np.random.default_rng(17)
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):   # two calls in a row share the static scratch
        f = rng.standard_normal((nz, ny, nx))
        spec = box.r2c(torch.from_numpy(f).to(box.device, box.rdtype))
        want = box.c2r(spec)
        got = torch.full_like(want, float("nan"))
        rc = lib.dnsbox_c2r_noalloc(nx, ny, nz, PRECISION[prec], ctypes.c_void_p(spec.data_ptr()),
                                    ctypes.c_void_p(got.data_ptr()), ctypes.c_void_p(stream))
        assert rc == 0, lib.dnsbox_last_error()
        torch.cuda.synchronize()
        assert _rel(got, want) < tol
    box.close()


def test_c2r_noalloc_rejects_oversize():
    from dnsbox_b200 import _lib
    lib = _lib.load()
    spec = torch.zeros(4, dtype=torch.complex128, device="cuda")
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    rc = lib.dnsbox_c2r_noalloc(128, 128, 128, 0, ctypes.c_void_p(spec.data_ptr()),
                                ctypes.c_void_p(out.data_ptr()), None)
    assert rc == -2
    assert b"scratch" in lib.dnsbox_last_error()
