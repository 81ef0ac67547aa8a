"""Time-horizon gradients on the GPU: the transpose of the fixed-dt IF-Heun
step, its checkpointed chain over many steps, and the periodic-orbit residual
J = 1/2 <|u(T) - u(0)|^2> of the adjoint configuration's periodic-orbit
variant (Kolmogorov forcing).

Bars: step transpose and orbit gradient against the oracle (FP64) within
1e-11 relative; directional derivatives against central finite differences of
the GPU's own forward steps (eps = 1e-6, FP64) within 1e-6; checkpointed
chains bit-identical for every checkpoint spacing."""
import numpy as np
import pytest
import torch

from oracle import dnsbox_oracle as O
from dnsbox_b200 import ic

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def ip(a, b):
    """Euclidean inner product on (Re, Im) of the half spectrum."""
    return float((a.real * b.real + a.imag * b.imag).sum())


def setup(n, prec="fp64", nu=1.0 / 40.0, dt=1e-2, seed=0):
    from dnsbox_b200.ops import Box
    b = Box(n, precision=prec, nu=nu, bandlim=False, tstep_fix=True, dt=dt, hminone=True)
    f = ic.kolmogorov_forcing(n, 1.0, 4)
    fd = b.from_numpy(f)
    b.set_forcing(fd)
    u = ic.random_field(n, seed=seed, k0=4.0, energy=0.5)
    return b, u, f, fd


def solenoidal(n, seed):
    g = O.Grid(O.Params(nx=n, ny=n, nz=n))
    rng = np.random.default_rng(seed)
    return O.state_dealias(g, O.state_project(g, O.state_u2uhat(g, rng.standard_normal((3, n, n, n)))))


def test_heun_step_vjp_matches_oracle():
    n, dt = 16, 1e-2
    b, u, f, _ = setup(n, dt=dt)
    g = O.Grid(O.Params(nx=n, ny=n, nz=n, nu=1.0 / 40.0, bandlim=False, tstep_fix=True))
    gout = solenoidal(n, 3) * 1e-3
    want = O.heun_step_vjp(g, u, dt, gout, f)
    got = b.heun_step_vjp(b.from_numpy(u), b.from_numpy(gout)).cpu().numpy()
    assert rel(got, want) < 1e-11
    # the forward step with the fixed forcing agrees with the oracle's too
    uu = b.from_numpy(u)
    b.step(uu, 1, diag=False)
    assert rel(uu.cpu().numpy(), O.heun_step(g, u, dt, f)) < 1e-12


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_heun_step_vjp_finite_differences(seed):
    """<S'(u)^T g, d> against (<g, S(u + eps d)> - <g, S(u - eps d)>) / (2 eps)
    with the GPU's own fused step."""
    n, dt, eps = 24, 1e-2, 1e-6
    b, u, _, _ = setup(n, dt=dt)
    d = solenoidal(n, 100 + seed)
    d /= np.sqrt(ip(d, d) / ip(u, u))
    gout = solenoidal(n, 200 + seed)
    lhs = ip(b.heun_step_vjp(b.from_numpy(u), b.from_numpy(gout)).cpu().numpy(), d)

    def fwd(x):
        t = b.from_numpy(x)
        b.step(t, 1, diag=False)
        return ip(gout, t.cpu().numpy())
    fd = (fwd(u + eps * d) - fwd(u - eps * d)) / (2 * eps)
    assert abs(lhs - fd) <= 1e-6 * abs(fd)


def test_orbit_residual_matches_oracle():
    n, dt, ns = 16, 1e-2, 8
    b, u, f, _ = setup(n, dt=dt)
    g = O.Grid(O.Params(nx=n, ny=n, nz=n, nu=1.0 / 40.0, bandlim=False, tstep_fix=True))
    Jw, gw = O.orbit_residual_grad(g, u, dt, ns, f)
    J, gr = b.orbit_residual(b.from_numpy(u), ns, every=3)
    assert abs(J - Jw) <= 1e-12 * Jw
    assert rel(gr.cpu().numpy(), gw) < 1e-11


def test_orbit_checkpoint_spacing_is_exact():
    """Recomputation from checkpoints reproduces the stored trajectory bit for
    bit, so the gradient does not depend on the checkpoint spacing."""
    n, ns = 24, 40
    b, u, _, _ = setup(n)
    u0 = b.from_numpy(u)
    J1, g1 = b.orbit_residual(u0, ns, every=1)
    for every in (7, 32, 40, 64):
        J, gr = b.orbit_residual(u0, ns, every=every)
        assert J == J1 and torch.equal(gr, g1)


@pytest.mark.parametrize("seed", [5, 6])
def test_orbit_gradient_finite_differences(seed):
    n, ns, eps = 16, 30, 1e-6
    b, u, _, _ = setup(n)
    J, gr = b.orbit_residual(b.from_numpy(u), ns, every=8)
    d = solenoidal(n, 300 + seed)
    d /= np.sqrt(ip(d, d) / ip(u, u))
    lhs = ip(gr.cpu().numpy(), d)
    Jp = b.orbit_residual(b.from_numpy(u + eps * d), ns, grad=False)
    Jm = b.orbit_residual(b.from_numpy(u - eps * d), ns, grad=False)
    fd = (Jp - Jm) / (2 * eps)
    assert abs(lhs - fd) <= 1e-6 * abs(fd)


def test_heun_steps_autograd():
    """torch.autograd through heun_steps gives the chain transpose."""
    from dnsbox_b200.autograd import heun_steps
    n, ns = 16, 12
    b, u, _, _ = setup(n)
    u0 = b.from_numpy(u).requires_grad_(True)
    w = b.from_numpy(solenoidal(n, 9))
    uT = heun_steps(b, u0, ns, every=5)
    loss = (w.conj() * uT).real.sum()
    loss.backward()
    want = b.heun_steps_vjp(b.from_numpy(u), ns, w, every=5)
    assert torch.equal(u0.grad, want)


def test_periodic_orbit_96():
    """Periodic-orbit variant of the adjoint configuration: 96^3, Kolmogorov
    forcing F = 1 at kf = 4, nu = 1/40, T = 5 (500 steps of dt = 1e-2),
    checkpoints every 32 steps, FP32 bulk with FP64 J.  The initial guess is
    the state after t = 5 from a seeded k0 = 4 field.  A step along -grad
    with backtracking lowers J, and the directional derivative agrees with
    the FP64-accumulated J differences along the same direction."""
    n, ns = 96, 500
    b, u, _, _ = setup(n, prec="fp32")
    x = b.from_numpy(u)
    b.step(x, ns, diag=False)
    J, gr = b.orbit_residual(x, ns, every=32)
    slope = float((gr.real.double() ** 2 + gr.imag.double() ** 2).sum())
    assert np.isfinite(J) and J > 0 and slope > 0
    alpha = 0.1 * J / slope
    for _ in range(20):
        Jt = b.orbit_residual(x - alpha * gr, ns, grad=False)
        if Jt < J - 1e-4 * alpha * slope:
            break
        alpha *= 0.5
    print(f"periodic orbit 96^3 T=5: J {J:.6e} -> {Jt:.6e} (alpha {alpha:.3e})")
    assert Jt < J
