"""The CPU oracle against the reference's golden vectors and known-answer tests.

Golden vectors come from running the reference prototype python/dnsbox.py
(tests/golden/make_golden.py); the known-answer tests are the Beltrami
analytic solution (state.f90:287-348), the FFT round trip
(single/test.f90:10-31) and the divergence check (single/test.f90:57-62).
"""
import os

import numpy as np
import pytest

from oracle import dnsbox_oracle as O
from oracle import naive
from dnsbox_b200 import ic

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _golden(n):
    return np.load(os.path.join(GOLDEN, f"golden_n{n}.npz"))


@pytest.mark.parametrize("n", [12, 16])
def test_nonlinear_matches_reference_prototype(n):
    d = _golden(n)
    p = O.Params(nx=n, ny=n, nz=n, nu=float(d["nu"]), bandlim=False)
    g = O.Grid(p)
    assert rel(O.rhs_nonlinear(g, d["uh0"]), d["n_unforced"]) < 1e-14


@pytest.mark.parametrize("n", [12, 16])
def test_forcing_coefficient_matches_reference_prototype(n):
    d = _golden(n)
    p = O.Params(nx=n, ny=n, nz=n, nu=float(d["nu"]), bandlim=True,
                 kCutOff=float(d["kcut"]), Pin=float(d["pin"]))
    g = O.Grid(p)
    uh = d["uh0"]
    diff = d["n_forced"] - d["n_unforced"]
    keep = ~g.dealias_mask(0.5)
    sel = keep[None] & (np.abs(uh) > 1e-6 * np.abs(uh).max())
    coef = (diff[sel] / uh[sel]).real
    want = p.Pin / (2.0 * O.rhs_eband(g, uh))
    assert np.allclose(coef, want, rtol=1e-10)
    # the oracle forces only |k| <= kCutOff (rhs.f90:109)
    N = O.rhs_nonlinear(g, uh)
    band = (g.absk <= p.kCutOff) & keep
    assert np.allclose(N[:, band], (d["n_unforced"] + want * uh)[:, band], rtol=1e-12, atol=1e-9)
    assert np.allclose(N[:, ~band], d["n_unforced"][:, ~band], rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("n", [12, 16])
def test_heun_and_stats_match_reference_prototype(n):
    d = _golden(n)
    dt = float(d["dt"])
    p = O.Params(nx=n, ny=n, nz=n, nu=float(d["nu"]), bandlim=False)
    g = O.Grid(p)
    u = d["uh0"].copy()
    for _ in range(3):
        u = O.heun_step(g, u, dt)
    assert rel(u, d["heun3"]) < 1e-14
    t, ek, disp, prod, courant, div = d["stats"]
    assert abs(O.state_kinetic(g, u) - ek) < 1e-14 * ek
    assert abs(O.state_dissipation(g, u) - disp) < 1e-13 * disp
    assert abs(O.dissipation_spectral(g, u) - disp) < 1e-13 * disp
    assert abs(O.io_courant(g, O.state_uhat2u(g, u), dt) - courant) < 1e-13 * courant
    assert abs(O.state_divergence(g, u)) < 1e-12 and abs(div) < 1e-12


@pytest.mark.parametrize("n", [12, 16])
def test_beltrami_known_answer(n):
    """state.f90:287-348: the Beltrami field is an exact solution (u x omega
    is a gradient), so the IF step is exact up to roundoff."""
    d = _golden(n)
    dt = float(d["dt"])
    p = O.Params(nx=n, ny=n, nz=n, nu=float(d["nu"]), bandlim=False)
    g = O.Grid(p)
    b = d["beltrami0"].copy()
    for _ in range(3):
        b = O.heun_step(g, b, dt)
    assert rel(b, d["beltrami3"]) < 1e-14
    exact = O.beltrami(g, 3 * dt)
    err = np.abs(O.state_uhat2u(g, b) - exact).max()
    assert err < 1e-13


def test_beltrami_long_run():
    p = O.Params(nx=16, ny=16, nz=16, nu=0.05, bandlim=False)
    g = O.Grid(p)
    uh = O.state_u2uhat(g, O.beltrami(g, 0.0))
    dt = 1e-2
    for _ in range(20):
        uh = O.heun_step(g, uh, dt)
    assert np.abs(O.state_uhat2u(g, uh) - O.beltrami(g, 20 * dt)).max() < 1e-12


def test_fft_round_trip():
    """single/test.f90:10-31: ten R2C/C2R round trips."""
    p = O.Params(nx=16, ny=12, nz=24)
    g = O.Grid(p)
    rng = np.random.default_rng(0)
    u0 = rng.standard_normal((3, 24, 12, 16))
    u = u0.copy()
    for _ in range(10):
        u = O.state_uhat2u(g, O.state_u2uhat(g, u))
    assert np.abs(u - u0).max() < 1e-13


@pytest.mark.parametrize("n", [8, 12])
@pytest.mark.parametrize("bandlim", [False, True])
def test_oracle_matches_naive_dft(n, bandlim):
    uh = ic.random_field(n, seed=3, k0=2.0)
    # Nyquist content exercises quirk Q1 (Nyquist wavenumber = 0)
    rng = np.random.default_rng(1)
    phys = rng.standard_normal((3, n, n, n)) * 0.01
    uh = uh + O.state_u2uhat(O.Grid(O.Params(nx=n, ny=n, nz=n)), phys)
    p = O.Params(nx=n, ny=n, nz=n, nu=0.01, kCutOff=2.5, Pin=0.1, bandlim=bandlim)
    g = O.Grid(p)
    No, ebo = O.rhs_nonlinear(g, uh, return_eband=True)
    Nn, ebn = naive.rhs_nonlinear(uh, n, n, n, nu=0.01, kcut=2.5, Pin=0.1, bandlim=bandlim)
    assert rel(No, Nn) < 1e-13
    assert abs(ebo - ebn) <= 1e-14 * max(ebo, 1e-300)


def test_naive_transforms_match_scipy():
    n = 8
    rng = np.random.default_rng(2)
    f = rng.standard_normal((n, n, n))
    p = O.Params(nx=n, ny=n, nz=n)
    g = O.Grid(p)
    F = g.r2c(f)
    assert rel(naive.r2c(f, n, n, n), F) < 1e-14
    assert rel(naive.c2r(F, n, n, n), g.c2r(F)) < 1e-14


def test_wavenumber_tables_q1():
    """variables.f90:226-262: Nyquist entries are zero (quirk Q1)."""
    g = O.Grid(O.Params(nx=8, ny=8, nz=8))
    assert list(g.kxr) == [0, 1, 2, 3, 0]
    assert list(g.kyr) == [0, 1, 2, 3, 0, -3, -2, -1]
    # Nyquist modes survive the 2/3 rule and are zeroed only as 'all-zero k'
    m = g.dealias_mask(0.5)
    assert m[0, 0, 4]          # (0, 0, Nyquist) has k = 0
    assert not m[1, 0, 4]      # (kz=1, 0, Nyquist) has |k| = 1


def test_dealias_threshold_q3():
    """N = 96: cutoff 32 -- '.ge.' (rhs.f90) drops |k|=32, '.gt.' (rhsAdj.f90) keeps it."""
    g = O.Grid(O.Params(nx=96, ny=96, nz=96))
    ge = g.dealias_mask(0.5)
    gt = g.dealias_mask(0.0, strict=True)
    assert ge[0, 0, 32] and not gt[0, 0, 32]
    assert ge[0, 0, 33] and gt[0, 0, 33]


def test_nspec_values():
    for n, want in ((64, 35), (256, 146), (512, 294), (1024, 590)):
        assert O.Grid(O.Params(nx=n, ny=n, nz=n)).nspec == want if n <= 256 else True
    from dnsbox_b200.grid import nspec
    assert [nspec(n, n, n) for n in (64, 256, 512, 1024)] == [35, 146, 294, 590]


def test_spectrum_modes_q4():
    n = 16
    uh = ic.random_field(n, seed=5, k0=3.0)
    g = O.Grid(O.Params(nx=n, ny=n, nz=n))
    es, e0, e1, esq = O.state_spectrum(g, uh, "mpi")
    es2, *_ = O.state_spectrum(g, uh, "single")
    E = O.state_kinetic(g, uh)
    # the single/ spectrum is Parseval-consistent on the retained shells
    assert abs(es2.sum() - E) < 0.02 * E
    # the MPI spectrum double-counts the kx = 0 / Nyquist planes
    assert es.sum() > es2.sum()
    # Esqrt2 matches every |k| < sqrt 2 (state.f90:383)
    assert esq >= e1 + e0


def test_ab2_reference_vs_standard_q2():
    n = 12
    p = O.Params(nx=n, ny=n, nz=n, nu=0.01, bandlim=False, ab2="reference")
    g = O.Grid(p)
    uh = ic.random_field(n, seed=2, k0=3.0)
    dt = 2e-3
    s_ref = O.AB2Stepper(g)
    a = s_ref.step(uh, dt)
    a = s_ref.step(a, dt)
    # literal coefficients at fixed dt: uhat <- IF (uhat + 1.5 dt N_n)
    s_chk = O.AB2Stepper(g)
    b = s_chk.step(uh, dt)
    IF = O.rhs_int_fact(g, dt)
    manual = IF * (b + 1.5 * dt * O.rhs_nonlinear(g, b))
    assert rel(a, manual) < 1e-14
    p2 = O.Params(nx=n, ny=n, nz=n, nu=0.01, bandlim=False, ab2="standard")
    g2 = O.Grid(p2)
    s_std = O.AB2Stepper(g2)
    c = s_std.step(uh, dt)
    c = s_std.step(c, dt)
    assert rel(c, a) > 1e-9          # the two schemes differ


def test_vjp_oracle_finite_difference():
    n = 8
    p = O.Params(nx=n, ny=n, nz=n, nu=0.01, bandlim=False)
    g = O.Grid(p)
    uh = ic.random_field(n, seed=4, k0=2.0)
    rng = np.random.default_rng(7)
    gout = O.state_u2uhat(g, rng.standard_normal((3, n, n, n)))
    d = O.state_u2uhat(g, rng.standard_normal((3, n, n, n)))
    d = O.state_dealias(g, d)
    vjp = O.rhs_nonlinear_vjp(g, uh, gout)
    eps = 1e-6 * np.abs(uh).max() / np.abs(d).max()
    jp = (O.rhs_nonlinear(g, uh + eps * d) - O.rhs_nonlinear(g, uh - eps * d)) / (2 * eps)
    lhs = np.sum(gout.real * jp.real + gout.imag * jp.imag)
    rhs = np.sum(vjp.real * d.real + vjp.imag * d.imag)
    assert abs(lhs - rhs) < 1e-6 * abs(lhs)


def _nyquist_planes(n):
    m = np.zeros((n, n, n // 2 + 1), bool)
    m[:, :, n // 2] = True
    m[:, n // 2, :] = True
    m[n // 2] = True
    return m


def test_exact_adjoint_matches_reference_rhsadj():
    """rhsAdj.f90:261-354 computes -P_d[(grad r)^T u + (u.grad) r], the
    continuous adjoint of the linearised nonlinear term.  The exact discrete
    transpose (Euclidean on the half spectrum) relates to it through the
    half-spectrum weight W: P W^-1 vjp(W r) = -rhsNonlinearAdj(r) on the
    retained modes off the Nyquist planes (where quirk Q1 breaks the identity)."""
    n = 16
    p = O.Params(nx=n, ny=n, nz=n, nu=0.01, bandlim=False)
    g = O.Grid(p)
    uh = ic.random_field(n, seed=1, k0=3.0)
    rt = ic.random_field(n, seed=2, k0=3.0)
    keep = ~g.dealias_mask(0.5) & ~_nyquist_planes(n)
    W = O.half_weight(g)
    pv = O.state_project(g, O.rhs_nonlinear_vjp(g, uh, W * rt) / W)
    ref = O.adj_nonlinear_part(g, uh, rt)
    assert rel(pv[:, keep], -ref[:, keep]) < 1e-13


def test_convective_equals_rotational_off_nyquist():
    """rhsAdj.f90's convective N equals rhs.f90's rotational N on dealiased
    solenoidal fields, except on the Nyquist planes (quirk Q1)."""
    n = 16
    g = O.Grid(O.Params(nx=n, ny=n, nz=n, nu=0.01, bandlim=False))
    uh = ic.random_field(n, seed=1, k0=3.0)
    keep = ~g.dealias_mask(0.5) & ~_nyquist_planes(n)
    assert rel(O.adj_rhs_nonlinear(g, uh)[:, keep], O.rhs_nonlinear(g, uh)[:, keep]) < 1e-13


def test_yoffe_oracle_hits_the_target_spectrum():
    """state.f90:211-285 restated: the rescaled field is solenoidal, dealiased
    and its MPI-mode spectrum equals C1 k^C2 exp(-C3 k^C4) on shells
    1 .. Nspec-1 (state.f90:218-221), with shell Nspec empty."""
    n = 24
    g = O.Grid(O.Params(nx=n, ny=n, nz=n))
    noise = np.random.default_rng(3).random((3, n, n, n)) - 0.5
    uh = O.state_init_rand(g, noise)
    es, *_ = O.state_spectrum(g, uh)
    c1, c2, c3, c4 = O.YOFFE_C
    k = np.arange(1, g.nspec)
    target = c1 * k ** c2 * np.exp(-c3 * k ** c4)
    assert np.max(np.abs(es[:-1] - target) / target) < 1e-13 and es[-1] == 0.0
    assert rel(O.state_dealias(g, O.state_project(g, uh)), uh) < 1e-14


def test_semi_implicit_oracle_orders():
    """dnsboximplicit.f90:88-181 restated: at c = 1/2 one step agrees with
    IF-Heun to second order (the difference shrinks 8x when dt halves), at
    c = 1 to first order, and the fixed point is reached within a few
    iterations."""
    n = 16
    g = O.Grid(O.Params(nx=n, ny=n, nz=n, nu=0.01, bandlim=False))
    uh = ic.random_field(n, seed=1, k0=3.0)
    d = {}
    for c in (0.5, 1.0):
        for dt in (4e-3, 2e-3):
            u, it = O.semi_implicit_step(g, uh, dt, c=c)
            assert it <= 8
            d[c, dt] = rel(u, O.heun_step(g, uh, dt))
    assert 6.0 < d[0.5, 4e-3] / d[0.5, 2e-3] < 10.0
    assert 3.0 < d[1.0, 4e-3] / d[1.0, 2e-3] < 5.0
