"""torch.ops.dnsbox.* (the C++ operator library over the C ABI) against the
ctypes binding: the same library calls, so the same results bit for bit, and
autograd through rhs_nonlinear is the exact transpose."""
import numpy as np
import pytest
import torch

from dnsbox_b200 import ic

pytestmark = pytest.mark.gpu


def test_torch_ops_equal_the_ctypes_binding():
    from dnsbox_b200 import torch_ops
    from dnsbox_b200.ops import Box
    ops = torch_ops.load()
    n = 32
    b = Box(n, nu=0.01, kCutOff=2.5, Pin=0.1, bandlim=True, tstep_fix=True, dt=2e-3)
    u = b.from_numpy(ic.random_field(n, seed=2, k0=3.0))
    N1, _ = b.rhs_nonlinear(u)
    assert torch.equal(ops.rhs_nonlinear(b.handle, u), N1)
    g = b.from_numpy(ic.random_field(n, seed=3, k0=5.0))
    assert torch.equal(ops.rhs_nonlinear_vjp(b.handle, u, g), b.rhs_nonlinear_vjp(u, g))
    phys = b.c2r(u[0].contiguous())
    assert torch.equal(ops.c2r(b.handle, u[0].contiguous(), n), phys)
    assert torch.equal(ops.r2c(b.handle, phys), b.r2c(phys))
    v = u.clone()
    ops.step_(b.handle, v, 2)
    b.set_time(0.0)
    w = u.clone()
    b2 = Box(n, nu=0.01, kCutOff=2.5, Pin=0.1, bandlim=True, tstep_fix=True, dt=2e-3)
    b2.step(w, 2)
    assert torch.equal(v, w)
    b.close()
    b2.close()


def test_torch_ops_autograd_is_the_transpose():
    from dnsbox_b200 import torch_ops
    from dnsbox_b200.ops import Box
    ops = torch_ops.load()
    n = 16
    b = Box(n, nu=0.01, bandlim=False)
    u = b.from_numpy(ic.random_field(n, seed=7, k0=3.0)).requires_grad_(True)
    c = b.from_numpy(ic.random_field(n, seed=8, k0=5.0))
    N = ops.rhs_nonlinear(b.handle, u)
    loss = torch.sum(c.real * N.real + c.imag * N.imag)
    loss.backward()
    want = b.rhs_nonlinear_vjp(u.detach(), c)
    assert torch.equal(u.grad, want)
    b.close()
