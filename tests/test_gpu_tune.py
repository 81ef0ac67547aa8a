"""The kernel-schedule autotuner: every candidate schedule is parity-green
against the oracle, the tuned schedule is no slower than the default in the
tuning run, the caller's state and clock are untouched, and later contexts of
the same shape start with the cached choice."""
import numpy as np
import pytest
import torch

from oracle import dnsbox_oracle as O
from dnsbox_b200 import ic

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("prec", ["tc_split", "fp32"])
def test_every_schedule_matches_the_oracle(prec):
    from dnsbox_b200.ops import Box
    n = 256   # the size with all four x-pass kernels
    kw = dict(nu=2e-3, kCutOff=2.5, Pin=0.1, bandlim=True)
    uh = ic.random_field(n, seed=12, k0=3.0)
    want = O.rhs_nonlinear(O.Grid(O.Params(nx=n, ny=n, nz=n, **kw)), uh)
    b = Box(n, precision=prec, **kw)
    u = b.from_numpy(uh)
    # each kernel on each of passes A, B, D (TMA 0, cp.async 1, SIMT 2)
    tcs = [(0, 0, 0), (1, 1, 1), (2, 2, 2), (0, 1, 2), (2, 0, 1), (1, 2, 0)] if prec == "tc_split" else [(0, 0, 0)]
    for tc in tcs:
        for xk in (0, 1, 2, 3, 4):
            for zt in ((False, True) if prec == "tc_split" else (False,)):
                b.set_schedule(tc, xk, zt)
                got, _ = b.rhs_nonlinear(u)
                assert rel(got.cpu().numpy(), want) < 2e-6, (tc, xk, zt)
    b.close()


@pytest.mark.parametrize("prec", ["tc_split", "fp64"])
def test_autotune_keeps_state_clock_and_caches(prec):
    from dnsbox_b200.ops import Box
    n = 128
    kw = dict(nu=2e-3, kCutOff=2.5, Pin=0.1, bandlim=True, courant_min=0.5, courant_max=0.5)
    b = Box(n, precision=prec, **kw)
    u = b.from_numpy(ic.random_field(n, seed=3, k0=3.0))
    b.step(u, 2)
    t0, dt0 = b.get_time(), b.get_dt()
    u0 = u.clone()
    sch = b.autotune(u, nsteps=3)
    assert sch["tuned"] and sch["ms_tuned"] <= sch["ms_default"] * (1 + 1e-12)
    assert torch.equal(u, u0)
    assert b.get_time() == t0 and b.get_dt() == dt0
    assert b.schedule()["tc_kernel"] == sch["tc_kernel"] and b.schedule()["x_kernel"] == sch["x_kernel"]
    # stepping after tuning continues the trajectory of an untuned context
    c = Box(n, precision=prec, **kw)
    v = c.from_numpy(ic.random_field(n, seed=3, k0=3.0))
    c.step(v, 2)
    assert c.schedule()["tc_kernel"] == sch["tc_kernel"]   # the cached choice
    c.set_schedule((0, 0, 0), 0, False)
    b.step(u, 2)
    c.step(v, 2)
    assert rel(u.to(torch.complex128).cpu().numpy(), v.to(torch.complex128).cpu().numpy()) < (
        1e-13 if prec == "fp64" else 2e-6)
    b.close()
    c.close()



@pytest.mark.parametrize("prec", ["fp32", "fp64", "tc_split"])
@pytest.mark.parametrize("bandlim", [False, True])
@pytest.mark.parametrize("nx", [256, 512])
def test_x_kernels_on_a_rough_field(nx, prec, bandlim):
    """Every fused-x-pass kernel on a white-noise field, whose vorticity is
    larger than its velocity by the grid's wavenumbers (the kernels that
    transform a velocity and a vorticity line as one complex sequence must
    balance the two first), on boxes with short y and z extents: the x pass
    works line by line, so the shape covers it while the oracle stays quick."""
    from dnsbox_b200.ops import Box
    ny, nz = 12, 16
    kw = dict(nu=2e-3, kCutOff=2.5, Pin=0.1, bandlim=bandlim)
    g = O.Grid(O.Params(nx=nx, ny=ny, nz=nz, **kw))
    rng = np.random.default_rng(21)
    uh = O.state_dealias(g, O.state_project(g, O.state_u2uhat(g, rng.standard_normal((3, nz, ny, nx)))))
    want = O.rhs_nonlinear(g, uh)
    b = Box(nx=nx, ny=ny, nz=nz, precision=prec, **kw)
    u = b.from_numpy(uh)
    tol = 1e-12 if prec == "fp64" else 2e-6
    for xk in ("block", "warp", "warp-registers", "warp-registers-128"):
        b.set_schedule((1, 1, 1), xk, False)
        got, _ = b.rhs_nonlinear(u)
        assert rel(got.cpu().numpy(), want) < tol, xk
    b.close()
