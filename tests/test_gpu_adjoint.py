"""Adjoint operators on the GPU against the oracle, the reference's rhsAdj,
central finite differences and torch autograd."""
import numpy as np
import pytest
import torch

from oracle import dnsbox_oracle as O
from dnsbox_b200 import ic

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def box(n, precision="fp64", **kw):
    from dnsbox_b200.ops import Box
    return Box(n, precision=precision, **kw)


def edot(a, b):
    """Euclidean inner product on the Re/Im parts (torch's complex-gradient geometry)."""
    return float(torch.sum(a.real * b.real + a.imag * b.imag).item())


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 2e-5)])
@pytest.mark.parametrize("n", [16, 24, 32])
def test_vjp_matches_oracle(prec, tol, n):
    p = O.Params(nx=n, ny=n, nz=n, nu=0.01, bandlim=False)
    g = O.Grid(p)
    uh = ic.random_field(n, seed=n, k0=3.0)
    rng = np.random.default_rng(n)
    gout = O.state_u2uhat(g, rng.standard_normal((3, n, n, n)))
    want = O.rhs_nonlinear_vjp(g, uh, gout)
    b = box(n, prec, nu=0.01, bandlim=False)
    got = b.rhs_nonlinear_vjp(b.from_numpy(uh), b.from_numpy(gout)).cpu().numpy()
    assert rel(got, want) < tol


@pytest.mark.parametrize("bandlim", [False, True])
def test_vjp_finite_difference(bandlim):
    """<g, N'(u) d> = <vjp(g), d> with N' from central differences (FP64)."""
    n = 24
    b = box(n, nu=0.01, bandlim=bandlim, kCutOff=2.5, Pin=0.1)
    u = b.from_numpy(ic.random_field(n, seed=3, k0=3.0))
    gnp = np.random.default_rng(5)
    g = b.from_numpy(ic.random_field(n, seed=11, k0=5.0))
    for s in range(4):
        d = b.from_numpy(ic.random_field(n, seed=100 + s, k0=3.0))
        eps = 1e-6
        np_, _ = b.rhs_nonlinear(u + eps * d)
        nm_, _ = b.rhs_nonlinear(u - eps * d)
        lhs = edot(g, (np_ - nm_) / (2 * eps))
        rhs = edot(b.rhs_nonlinear_vjp(u, g), d)
        assert abs(lhs - rhs) <= 1e-7 * abs(rhs)
    del gnp


@pytest.mark.parametrize("n", [16, 24])
@pytest.mark.parametrize("phat", ["intent", "literal"])
@pytest.mark.parametrize("hminone", [True, False])
def test_rhs_adj_matches_oracle(n, phat, hminone):
    """rhsAdj.f90:356-381 literal (N = 24 has an integer 2/3 cutoff: quirk Q3)."""
    p = O.Params(nx=n, ny=n, nz=n, nu=0.02, Q=0.01, bandlim=False, hminone=hminone, adj_phat=phat)
    g = O.Grid(p)
    uh = ic.random_field(n, seed=2, k0=3.0)
    # add Nyquist and beyond-cutoff content so the '.gt.' mask and Q1 matter
    rng = np.random.default_rng(9)
    uh = uh + 1e-3 * O.state_u2uhat(g, rng.standard_normal((3, n, n, n)))
    rt_w, adj_w = O.rhs_adj(g, uh)
    b = box(n, nu=0.02, Q=0.01, bandlim=False, hminone=hminone, adj_phat=phat)
    rt, adj = b.rhs_adj(b.from_numpy(uh))
    assert rel(rt.cpu().numpy(), rt_w) < 1e-12
    assert rel(adj.cpu().numpy(), adj_w) < 1e-12


def test_exact_adjoint_equals_reference_rhsadj_term():
    """P W^-1 vjp(W r~) = -rhsNonlinearAdj(r~) (rhsAdj.f90:261-354) on the
    retained modes off the Nyquist planes."""
    n = 32
    p = O.Params(nx=n, ny=n, nz=n, nu=0.01, bandlim=False)
    g = O.Grid(p)
    uh = ic.random_field(n, seed=1, k0=3.0)
    rt = ic.random_field(n, seed=2, k0=3.0)
    W = O.half_weight(g)
    b = box(n, nu=0.01, bandlim=False)
    v = b.rhs_nonlinear_vjp(b.from_numpy(uh), b.from_numpy(W * rt)).cpu().numpy() / W
    pv = O.state_project(g, v)
    ref = O.adj_nonlinear_part(g, uh, rt)
    nyq = np.zeros(rt.shape[1:], bool)
    nyq[:, :, n // 2] = nyq[:, n // 2, :] = nyq[n // 2] = True
    keep = ~g.dealias_mask(0.5) & ~nyq
    assert rel(pv[:, keep], -ref[:, keep]) < 1e-12


def _kolmogorov_box(n, precision="fp64", hminone=True):
    b = box(n, precision, nu=1.0 / 40.0, bandlim=False, hminone=hminone, tstep_fix=True, dt=5e-3)
    f = b.from_numpy(ic.kolmogorov_forcing(n, 1.0, 4))
    b.set_forcing(f)
    return b


@pytest.mark.parametrize("n", [32, 64])
@pytest.mark.parametrize("hminone", [True, False])
def test_residual_gradient_finite_differences(n, hminone):
    """dJ along 16 seeded solenoidal directions, eps = 1e-6, FP64: the exact
    adjoint gradient agrees with central differences to 1e-6 (64^3 is the
    adjoint-descent configuration's grid)."""
    b = _kolmogorov_box(n, hminone=hminone)
    u = b.from_numpy(ic.random_field(n, seed=0, k0=4.0))
    J, grad = b.residual_grad(u)
    assert J > 0
    unorm = float(u.abs().norm())
    worst = 0.0
    for s in range(16):
        d = b.from_numpy(ic.random_field(n, seed=1000 + s, k0=4.0))
        d = d * (unorm / float(d.abs().norm()))
        eps = 1e-6
        fd = (b.residual(u + eps * d) - b.residual(u - eps * d)) / (2 * eps)
        an = edot(grad, d)
        worst = max(worst, abs(fd - an) / abs(an))
    assert worst < 1e-6, worst


def test_residual_matches_oracle():
    n = 24
    p = O.Params(nx=n, ny=n, nz=n, nu=1.0 / 40.0, bandlim=False, hminone=True)
    g = O.Grid(p)
    uh = ic.random_field(n, seed=4, k0=4.0)
    f = ic.kolmogorov_forcing(n, 1.0, 4)
    mask = g.dealias_mask(0.5)
    N = O.rhs_nonlinear(g, uh) + np.where(mask[None], 0.0, f)
    kk = np.real(g.kx * g.kx + g.ky * g.ky + g.kz * g.kz)
    r = (p.nu * kk + p.Q) * uh + N
    W = O.half_weight(g)
    h = 1.0 / (1.0 - kk)
    Jw = 0.5 * g.scalemodes ** 2 * float(np.sum(W * h * np.abs(r) ** 2))
    b = _kolmogorov_box(n)
    assert abs(b.residual(b.from_numpy(uh)) - Jw) < 1e-12 * Jw


def test_autograd_backward_is_the_adjoint():
    from dnsbox_b200.autograd import rhs_nonlinear, residual
    n = 16
    b = box(n, nu=0.01, bandlim=False)
    u = b.from_numpy(ic.random_field(n, seed=7, k0=3.0)).requires_grad_(True)
    c = b.from_numpy(ic.random_field(n, seed=8, k0=5.0))
    N = rhs_nonlinear(b, u)
    loss = torch.sum(c.real * N.real + c.imag * N.imag)
    loss.backward()
    want = b.rhs_nonlinear_vjp(u.detach(), c)
    assert float((u.grad - want).abs().max()) <= 1e-14 * float(want.abs().max())
    # J through autograd equals residual_grad
    kb = _kolmogorov_box(n)
    v = kb.from_numpy(ic.random_field(n, seed=9, k0=4.0)).requires_grad_(True)
    J = residual(kb, v)
    J.backward()
    J2, g2 = kb.residual_grad(v.detach())
    assert abs(J.item() - J2) < 1e-14 * J2
    assert float((v.grad - g2).abs().max()) <= 1e-14 * float(g2.abs().max())


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_adjoint_descent_graph_reuse_is_exact(prec):
    """The descent iterations run as captured graph launches (two buffer
    parities, cached per state tensor).  One call of seven iterations equals
    seven calls of one (graphs reused across calls, the parity restarting at
    each call) bit for bit, on a second state tensor whose new pointer makes
    the cache capture its graphs again."""
    n = 32
    b = _kolmogorov_box(n, prec)
    u0 = ic.random_field(n, seed=4, k0=4.0)
    ua = b.from_numpy(u0)
    ha, aa = b.adjoint_descent(ua, 7, alpha=1.0)
    ub = b.from_numpy(u0)
    alpha, hb = 1.0, [ha[0]]
    for _ in range(7):
        h, alpha = b.adjoint_descent(ub, 1, alpha=alpha)
        assert h[0] == hb[-1]
        hb.append(h[1])
    assert np.array_equal(np.asarray(hb), ha) and alpha == aa
    assert torch.equal(ua, ub)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_adjoint_descent_decreases_J(prec):
    n = 32
    b = _kolmogorov_box(n, prec)
    u = b.from_numpy(ic.random_field(n, seed=3, k0=4.0))
    hist, alpha = b.adjoint_descent(u, 25, alpha=1.0)
    h = hist[np.isfinite(hist)]
    assert len(h) >= 20
    assert np.all(np.diff(h) <= 1e-12 * h[0])
    assert h[-1] < 0.9 * h[0]
    # the state stays solenoidal and dealiased
    assert b.divergence(u) < (1e-9 if prec == "fp64" else 1e-3)


def test_residual_gradient_tc_split_128():
    """The residual and its gradient with the tensor-core passes (128^3,
    Kolmogorov forcing; the transpose's C2R and R2C jobs run the tensor-core
    strided kernel too) against the FP64 form on the same state: J within
    1e-5 and the gradient within 2e-5 relative L2."""
    n = 128
    u0 = ic.random_field(n, seed=12, k0=4.0)
    res = {}
    for prec in ("fp64", "tc_split"):
        b = _kolmogorov_box(n, prec)
        J, g = b.residual_grad(b.from_numpy(u0))
        res[prec] = (J, g.to(torch.complex128).cpu())
        b.close()
    J64, g64 = res["fp64"]
    Jtc, gtc = res["tc_split"]
    eg = float((gtc - g64).abs().norm() / g64.abs().norm())
    print(f"tc_split residual 128^3: J {abs(Jtc - J64) / J64:.2e}, gradient {eg:.2e}")
    assert abs(Jtc - J64) <= 1e-5 * J64
    assert eg < 2e-5


def test_batched_context_refuses_residual_and_adjoint():
    """The adjoint arena holds one box: every residual and adjoint entry
    refuses a batched context with DNSBOX_ERR_UNSUPPORTED before launching."""
    from dnsbox_b200._lib import DnsboxError
    n = 16
    b = box(n, nu=0.01, bandlim=False, tstep_fix=True, nbatch=3)
    u = b.zeros()
    calls = [lambda: b.residual(u), lambda: b.residual_grad(u), lambda: b.rhs_adj(u),
             lambda: b.rhs_nonlinear_vjp(u, u), lambda: b.adjoint_descent(u, 1)]
    for call in calls:
        with pytest.raises(DnsboxError) as e:
            call()
        assert e.value.code == -8 and "batched" in str(e.value)
    b.close()


def test_adjoint_descent_follows_a_forcing_change():
    """The descent graphs capture the forcing pointer: after set_forcing the
    next descent on the same state tensor recaptures, and its J history equals
    that of a fresh context created with the new forcing."""
    n = 24
    b = _kolmogorov_box(n)
    u = b.from_numpy(ic.random_field(n, seed=5, k0=4.0))
    b.adjoint_descent(u, 2, alpha=1.0)
    f2 = b.from_numpy(2.0 * ic.kolmogorov_forcing(n, 1.0, 4))
    b.set_forcing(f2)
    u_after = u.clone()
    h, a = b.adjoint_descent(u, 3, alpha=1.0)
    c = _kolmogorov_box(n)
    c.set_forcing(c.from_numpy(2.0 * ic.kolmogorov_forcing(n, 1.0, 4)))
    v = u_after.clone()
    hc, ac = c.adjoint_descent(v, 3, alpha=1.0)
    assert np.array_equal(h, hc) and a == ac
    assert torch.equal(u, v)
