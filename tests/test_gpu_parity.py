"""GPU parity: libdnsbox_gpu.so (through the C ABI) against the CPU oracle.

Bars: FP64 within 1e-12 relative L2 (the north-star bar for the plain form);
FP32 within the single-precision tolerances written beside each case."""
import os

import numpy as np
import pytest
import torch

from oracle import dnsbox_oracle as O
from dnsbox_b200 import ic

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FP64_TOL = 1e-12
FP32_TOL = 2e-6   # one FP32 right-hand side measures 3-6e-7 against the FP64 oracle


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def box(n, precision="fp64", **kw):
    from dnsbox_b200.ops import Box
    return Box(n, precision=precision, **kw)


def field(n, seed, k0=3.0, nyquist=True):
    uh = ic.random_field(n, seed=seed, k0=k0)
    if nyquist:   # small broadband content, Nyquist planes included (quirk Q1)
        g = O.Grid(O.Params(nx=n, ny=n, nz=n))
        rng = np.random.default_rng(seed + 100)
        uh = uh + 1e-3 * O.state_u2uhat(g, rng.standard_normal((3, n, n, n)))
    return uh


def tol(prec):
    return FP64_TOL if prec == "fp64" else FP32_TOL


# ---------------------------------------------------------------- transforms
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("shape", [(8, 8, 8), (12, 12, 12), (16, 12, 24), (32, 48, 16), (64, 64, 64),
                                   (96, 96, 96), (128, 32, 64)])
def test_transforms_match_pocketfft(prec, shape):
    nx, ny, nz = shape
    from dnsbox_b200.ops import Box
    b = Box(nx=nx, ny=ny, nz=nz, precision=prec)
    g = O.Grid(O.Params(nx=nx, ny=ny, nz=nz))
    rng = np.random.default_rng(1)
    f = rng.standard_normal((nz, ny, nx))
    F = g.r2c(f)
    Fg = b.r2c(torch.from_numpy(f).to(b.device, b.rdtype)).cpu().numpy()
    assert rel(Fg, F) < (1e-13 if prec == "fp64" else 8e-7)   # FP32 measures 1-3e-7
    fg = b.c2r(torch.from_numpy(F).to(b.device, b.cdtype)).cpu().numpy()
    assert rel(fg, g.c2r(F)) < (1e-13 if prec == "fp64" else 8e-7)


@pytest.mark.parametrize("n", [256, 512])
def test_transform_round_trip_large(n):
    b = box(n)
    rng = torch.Generator(device="cuda").manual_seed(0)
    f = torch.randn((n, n, n), dtype=torch.float64, device=b.device, generator=rng)
    back = b.c2r(b.r2c(f)) / float(n) ** 3
    assert (back - f).abs().max().item() < 1e-12
    # against torch.fft on the device (cuFFT) as a library cross-check
    ref = torch.fft.rfftn(f, dim=(0, 1, 2))
    got = b.r2c(f)
    assert ((got - ref).abs().max() / ref.abs().max()).item() < 1e-13


# ---------------------------------------------------------------- nonlinear term
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("n", [8, 12, 16, 24, 32, 48, 64, 96, 128, 192])
@pytest.mark.parametrize("bandlim", [False, True])
def test_rhs_nonlinear(prec, n, bandlim):
    uh = field(n, seed=n, k0=3.0)
    p = O.Params(nx=n, ny=n, nz=n, nu=0.01, kCutOff=2.5, Pin=0.1, bandlim=bandlim)
    g = O.Grid(p)
    want, eb = O.rhs_nonlinear(g, uh, return_eband=True)
    b = box(n, prec, nu=0.01, kCutOff=2.5, Pin=0.1, bandlim=bandlim)
    got, ebg = b.rhs_nonlinear(b.from_numpy(uh))
    assert rel(got.cpu().numpy(), want) < tol(prec)
    if bandlim:
        assert abs(ebg - eb) < (1e-13 if prec == "fp64" else 1e-6) * eb


def test_rhs_nonlinear_noncubic_and_alpha():
    nx, ny, nz = 32, 16, 24
    p = O.Params(nx=nx, ny=ny, nz=nz, nu=0.01, kCutOff=3.0, Pin=0.2, bandlim=True,
                 alpha_x=1.0, alpha_y=2.0, alpha_z=0.5)
    g = O.Grid(p)
    rng = np.random.default_rng(3)
    uh = O.state_dealias(g, O.state_project(g, O.state_u2uhat(g, rng.standard_normal((3, nz, ny, nx)))))
    from dnsbox_b200.ops import Box
    b = Box(nx=nx, ny=ny, nz=nz, nu=0.01, kCutOff=3.0, Pin=0.2, alpha=(1.0, 2.0, 0.5))
    got, _ = b.rhs_nonlinear(b.from_numpy(uh))
    assert rel(got.cpu().numpy(), O.rhs_nonlinear(g, uh)) < FP64_TOL


@pytest.mark.parametrize("n", [12, 16])
def test_golden_vectors_on_gpu(n):
    """The GPU path against the reference prototype's own outputs."""
    d = np.load(os.path.join(GOLDEN, f"golden_n{n}.npz"))
    b = box(n, nu=float(d["nu"]), bandlim=False, tstep_fix=True, dt=float(d["dt"]))
    got, _ = b.rhs_nonlinear(b.from_numpy(d["uh0"]))
    assert rel(got.cpu().numpy(), d["n_unforced"]) < FP64_TOL
    u = b.from_numpy(d["uh0"])
    recs = b.step(u, 3)
    assert rel(u.cpu().numpy(), d["heun3"]) < FP64_TOL
    t, ek, disp, prod, courant, div = d["stats"]
    assert abs(recs[-1]["ekin"] - ek) < 1e-13 * ek
    assert abs(recs[-1]["dissipation"] - disp) < 1e-12 * disp
    assert abs(recs[-1]["t"] - t) < 1e-15
    c, _ = b.courant(u, float(d["dt"]))
    assert abs(c - courant) < 1e-12 * courant
    bel = b.from_numpy(d["beltrami0"])
    b.step(bel, 3)
    assert rel(bel.cpu().numpy(), d["beltrami3"]) < FP64_TOL


# ---------------------------------------------------------------- steppers
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("bandlim", [False, True])
def test_heun_steps(prec, bandlim):
    n, dt, ns = 32, 2e-3, 6
    uh = field(n, seed=11, k0=3.0)
    p = O.Params(nx=n, ny=n, nz=n, nu=0.01, kCutOff=2.5, Pin=0.1, bandlim=bandlim, tstep_fix=True)
    g = O.Grid(p)
    want, recs = O.drive(g, uh, ns, dt)
    b = box(n, prec, nu=0.01, kCutOff=2.5, Pin=0.1, bandlim=bandlim, tstep_fix=True, dt=dt)
    u = b.from_numpy(uh)
    grec = b.step(u, ns)
    assert rel(u.cpu().numpy(), want) < tol(prec) * (1 if prec == "fp64" else 2)
    for a, r in zip(grec, recs):
        assert abs(a["ekin"] - r["ekin"]) < (1e-12 if prec == "fp64" else 1e-5) * r["ekin"]
        assert abs(a["dissipation"] - r["dissipation"]) < (1e-12 if prec == "fp64" else 1e-5) * r["dissipation"]
        assert abs(a["courant"] - r["courant"]) < (1e-12 if prec == "fp64" else 1e-5) * r["courant"]
        assert a["dt"] == dt


@pytest.mark.parametrize("ab2", ["reference", "standard"])
def test_ab2_steps(ab2):
    n, dt, ns = 24, 2e-3, 8
    uh = field(n, seed=5, k0=3.0)
    p = O.Params(nx=n, ny=n, nz=n, nu=0.01, bandlim=False, ab2=ab2, tstep_fix=True)
    g = O.Grid(p)
    want, _ = O.drive(g, uh, ns, dt, stepper="ab2")
    b = box(n, nu=0.01, bandlim=False, stepper="ab2", ab2=ab2, tstep_fix=True, dt=dt)
    u = b.from_numpy(uh)
    b.step(u, 3)
    b.step(u, ns - 3)            # history carries across calls
    assert rel(u.cpu().numpy(), want) < FP64_TOL


@pytest.mark.parametrize("stepper", ["heun", "ab2"])
def test_cfl_controlled_steps(stepper):
    n, ns = 32, 6
    uh = field(n, seed=9, k0=3.0)
    kw = dict(nu=2e-3, kCutOff=2.5, Pin=0.1, bandlim=True, courant_min=0.5, courant_max=0.5, dt_max=1e-2)
    p = O.Params(nx=n, ny=n, nz=n, ab2="standard", **kw)
    g = O.Grid(p)
    want, recs = O.drive(g, uh, ns, 1e-3, stepper=stepper, cfl=True)
    b = box(n, stepper=stepper, ab2="standard", dt=1e-3, **kw)
    u = b.from_numpy(uh)
    grec = b.step(u, ns)
    assert rel(u.cpu().numpy(), want) < FP64_TOL
    for a, r in zip(grec, recs):
        assert abs(a["dt"] - r["dt"]) < 1e-13 * r["dt"]
        # 0.5 unless the dt cap (tStepMax) holds it below
        assert abs(a["courant"] - r["courant"]) < 1e-12 * r["courant"]
        assert r["courant"] <= 0.5 + 1e-12


def test_beltrami_known_answer_gpu():
    """state.f90:287-348 on the GPU: error at roundoff after many steps."""
    n, nu, dt = 32, 0.05, 1e-2
    g = O.Grid(O.Params(nx=n, ny=n, nz=n, nu=nu))
    b = box(n, nu=nu, bandlim=False, tstep_fix=True, dt=dt)
    u = b.zeros()
    b.upload_physical(ic.beltrami(n, nu, 0.0), u)
    b.step(u, 50)
    phys = b.download_physical(u)
    assert np.abs(phys - ic.beltrami(n, nu, 50 * dt)).max() < 1e-12


# ---------------------------------------------------------------- diagnostics
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_diagnostics(prec):
    n = 32
    uh = field(n, seed=21, k0=4.0)
    p = O.Params(nx=n, ny=n, nz=n, nu=0.01, kCutOff=2.5)
    g = O.Grid(p)
    b = box(n, prec, nu=0.01, kCutOff=2.5)
    u = b.from_numpy(uh)
    t = 1e-12 if prec == "fp64" else 1e-5
    assert abs(b.kinetic(u) - O.state_kinetic(g, uh)) < t * O.state_kinetic(g, uh)
    assert abs(b.dissipation(u) - O.state_dissipation(g, uh)) < t * O.state_dissipation(g, uh)
    assert abs(b.eband(u) - O.rhs_eband(g, uh)) < t * O.rhs_eband(g, uh)
    es, e0, e1, esq = b.spectrum(u)
    wes, we0, we1, wesq = O.state_spectrum(g, uh, "mpi")
    assert rel(es, wes) < t and abs(e1 - we1) < t * we1 and abs(esq - wesq) < t * wesq
    c, m = b.courant(u, 1e-3)
    assert abs(c - O.io_courant(g, O.state_uhat2u(g, uh), 1e-3)) < t * c
    assert abs(b.divergence(u) - O.state_divergence(g, uh)) < (1e-12 if prec == "fp64" else 1e-5)
    b2 = box(n, prec, spectrum_mode="single")
    es2, *_ = b2.spectrum(u)
    assert rel(es2, O.state_spectrum(g, uh, "single")[0]) < t


def test_project_dealias():
    n = 24
    g = O.Grid(O.Params(nx=n, ny=n, nz=n))
    rng = np.random.default_rng(4)
    uh = O.state_u2uhat(g, rng.standard_normal((3, n, n, n)))
    b = box(n)
    u = b.from_numpy(uh)
    b.project(u)
    assert rel(u.cpu().numpy(), O.state_project(g, uh)) < FP64_TOL
    b.dealias(u)
    assert rel(u.cpu().numpy(), O.state_dealias(g, O.state_project(g, uh))) < FP64_TOL


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_host_layout_round_trips(prec):
    n = 16
    uh = field(n, seed=2)
    b = box(n, prec)
    u = b.zeros()
    host = np.ascontiguousarray(np.transpose(uh, (0, 3, 2, 1)))   # p3dfft (kz fastest)
    b.upload_state(host, u)
    assert rel(u.cpu().numpy(), uh) < (1e-15 if prec == "fp64" else 1e-7)
    back = b.download_state(u)
    assert rel(back, host) < (1e-15 if prec == "fp64" else 1e-7)
    g = O.Grid(O.Params(nx=n, ny=n, nz=n))
    phys = b.download_physical(u)
    assert rel(phys, O.state_uhat2u(g, uh)) < (1e-13 if prec == "fp64" else 8e-7)
    u2 = b.zeros()
    b.upload_physical(phys, u2)
    assert rel(u2.cpu().numpy(), uh) < (1e-13 if prec == "fp64" else 8e-7)


# ---------------------------------------------------------------- full size
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_full_size_properties(prec):
    """256^3 forced turbulence (the benchmark workload): size-independent checks."""
    n = 256
    b = box(n, prec, nu=2e-3, kCutOff=2.5, Pin=0.1, courant_min=0.5, courant_max=0.5)
    u = b.from_numpy(ic.random_field(n, seed=0, k0=3.0))
    N, eb = b.rhs_nonlinear(u)
    # solenoidal and dealiased output
    from dnsbox_b200.grid import broadcast_k
    kz, ky, kx = [torch.from_numpy(np.ascontiguousarray(np.broadcast_to(k, (n, n, n // 2 + 1)))).to(b.device)
                  for k in broadcast_k(n, n, n)]
    kdot = (kx * N[0] + ky * N[1] + kz * N[2]).abs().max().item()
    assert kdot < (1e-9 if prec == "fp64" else 1e-2) * N.abs().max().item() * n
    cut = (kx.abs() >= n / 3) | (ky.abs() >= n / 3) | (kz.abs() >= n / 3)
    assert N[:, cut].abs().max().item() == 0.0
    # energy budget over a few steps: dE/dt = Pin - D (+ time-stepping error)
    recs = b.step(u, 10)
    e0 = b.kinetic(b.from_numpy(ic.random_field(n, seed=0, k0=3.0)))
    es = [e0] + [r["ekin"] for r in recs]
    for i, r in enumerate(recs):
        dEdt = (es[i + 1] - es[i]) / r["dt"]
        ds = recs[i - 1]["dissipation"] if i else None
        if ds is not None:
            assert abs(dEdt - (0.1 - 0.5 * (ds + r["dissipation"]))) < 0.02
    assert all(abs(r["courant"] - 0.5) < 1e-6 for r in recs[1:])


@pytest.mark.slow
@pytest.mark.parametrize("ab2", ["reference", "standard"])
def test_config0_parity(ab2):
    """64^3 decaying turbulence, IF-AB2 with a PC first step, dt = 2e-3, 200
    steps: final spectral velocity, E(k) and D every step within 1e-12."""
    n, dt, ns = 64, 2e-3, 200
    uh = ic.random_field(n, seed=0, k0=4.0)
    p = O.Params(nx=n, ny=n, nz=n, nu=0.01, bandlim=False, ab2=ab2, tstep_fix=True)
    g = O.Grid(p)
    want, recs = O.drive(g, uh, ns, dt, stepper="ab2")
    b = box(n, nu=0.01, bandlim=False, stepper="ab2", ab2=ab2, tstep_fix=True, dt=dt)
    u = b.from_numpy(uh)
    grec = b.step(u, ns)
    assert rel(u.cpu().numpy(), want) < FP64_TOL
    assert max(abs(a["dissipation"] - r["dissipation"]) / r["dissipation"] for a, r in zip(grec, recs)) < FP64_TOL
    es, *_ = b.spectrum(u)
    wes = O.state_spectrum(g, want, "mpi")[0]
    assert rel(es, wes) < FP64_TOL


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_gpu_initial_condition(prec):
    """Device IC: solenoidal, dealiased, Nyquist-free, E = 0.5, E(k) ~ k^4 exp(-2k^2/k0^2)."""
    from dnsbox_b200.ic import random_field_gpu
    n = 64
    b = box(n, prec)
    u = random_field_gpu(b, seed=5, k0=3.0)
    assert abs(b.kinetic(u) - 0.5) < (1e-12 if prec == "fp64" else 1e-6)
    assert abs(b.divergence(u)) < (1e-10 if prec == "fp64" else 1e-3)
    assert float(u[:, :, :, n // 2].abs().max()) == 0.0
    es, *_ = b.spectrum(u)
    k = np.arange(1, len(es) + 1, dtype=float)
    shape = k ** 4 * np.exp(-2 * k ** 2 / 9.0)
    ratio = es[:6] / shape[:6]
    assert np.all(np.abs(ratio / ratio[2] - 1) < 0.6)   # MPI spectrum: kx=0 planes double counted


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_rhs_nonlinear_256(prec):
    n = 256
    uh = ic.random_field(n, seed=2, k0=3.0)
    p = O.Params(nx=n, ny=n, nz=n, nu=2e-3, kCutOff=2.5, Pin=0.1, bandlim=True)
    want = O.rhs_nonlinear(O.Grid(p), uh)
    b = box(n, prec, nu=2e-3, kCutOff=2.5, Pin=0.1, bandlim=True)
    got, _ = b.rhs_nonlinear(b.from_numpy(uh))
    assert rel(got.cpu().numpy(), want) < tol(prec)


def test_rhs_nonlinear_512_properties():
    """512^3: the unforced rotational term conserves energy, <uhat, N(uhat)> = 0
    (W-weighted over the half spectrum), and FP32 agrees with FP64."""
    from dnsbox_b200.ic import random_field_gpu
    n = 512
    b64 = box(n, "fp64", bandlim=False)
    u64 = random_field_gpu(b64, seed=1, k0=3.0)
    N64, _ = b64.rhs_nonlinear(u64)
    W = torch.full((n // 2 + 1,), 2.0, dtype=torch.float64, device=u64.device)
    W[0] = W[n // 2] = 1.0
    dot = float((W * (u64.conj() * N64).real).sum())
    norm = float(u64.abs().norm() * N64.abs().norm())
    assert abs(dot) < 1e-12 * norm
    host = u64.cpu()
    del N64
    b64.close()
    b32 = box(n, "fp32", bandlim=False)
    u32 = host.to(b32.device, torch.complex64)
    N32, _ = b32.rhs_nonlinear(u32)
    b32.close()
    b64 = box(n, "fp64", bandlim=False)
    N64, _ = b64.rhs_nonlinear(host.to(b64.device))
    assert float((N32.to(torch.complex128) - N64).abs().norm() / N64.abs().norm()) < 2e-6


# ---------------------------------------------------------------- 512- and 1024-point axes
@pytest.mark.parametrize("prec", ["fp64", "fp32", "tc_split"])
@pytest.mark.parametrize("shape", [(1024, 16, 16), (16, 1024, 16), (16, 16, 1024), (16, 512, 24), (24, 16, 512)])
def test_long_axes(prec, shape):
    """Every pass at its largest sizes on small boxes (one axis of 512 or
    1024, where the FP32 strided kernel splits a tile over two CTAs): the
    transforms against pocketfft and one right-hand side against the oracle."""
    nx, ny, nz = shape
    from dnsbox_b200.ops import Box
    b = Box(nx=nx, ny=ny, nz=nz, precision=prec, nu=0.01, kCutOff=2.5, Pin=0.1, bandlim=True)
    p = O.Params(nx=nx, ny=ny, nz=nz, nu=0.01, kCutOff=2.5, Pin=0.1, bandlim=True)
    g = O.Grid(p)
    rng = np.random.default_rng(11)
    f = rng.standard_normal((nz, ny, nx))
    F = g.r2c(f)
    t = 1e-13 if prec == "fp64" else 2e-6
    assert rel(b.r2c(torch.from_numpy(f).to(b.device, b.rdtype)).cpu().numpy(), F) < t
    assert rel(b.c2r(torch.from_numpy(F).to(b.device, b.cdtype)).cpu().numpy(), g.c2r(F)) < t
    uh = O.state_dealias(g, O.state_project(g, O.state_u2uhat(g, rng.standard_normal((3, nz, ny, nx)))))
    got, _ = b.rhs_nonlinear(b.from_numpy(uh))
    assert rel(got.cpu().numpy(), O.rhs_nonlinear(g, uh)) < tol("fp64" if prec == "fp64" else "fp32")


def test_config1_500_steps_fp64_and_fp32():
    """Config 1 as specified: 256^3 forced turbulence (k0 = 3, band forcing
    0 < |k| <= 2.5 with Pin = 0.1, nu = 2e-3, Courant 0.5), 500 steps in the
    FP64 and the FP32 forms from the same seeded field.  Both close the energy
    budget dE/dt = Pin - D (trapezoidal D) to 1e-3 on every step after the
    first and hold the Courant number at 0.5; the reported production is the
    injected power Pin.  The two forms' dissipation series agree to 1e-3 and
    the final E(k) to 1e-2 on shells holding at least 1e-9 of the energy (the
    flow is chaotic over 500 steps, so FP32 round-off grows; the velocity
    difference is printed)."""
    n, ns = 256, 500
    kw = dict(nu=2e-3, kCutOff=2.5, Pin=0.1, courant_min=0.5, courant_max=0.5)
    uh = ic.random_field(n, seed=0, k0=3.0)
    out = {}
    for prec in ("fp64", "fp32"):
        b = box(n, prec, **kw)
        u = b.from_numpy(uh)
        e0 = b.kinetic(u)
        recs = b.step(u, ns)
        es, *_ = b.spectrum(u)
        E = [e0] + [r["ekin"] for r in recs]
        resid = max(abs((E[i + 1] - E[i]) / recs[i]["dt"]
                        - (0.1 - 0.5 * (recs[i - 1]["dissipation"] + recs[i]["dissipation"])))
                    for i in range(1, ns))
        assert resid < 1e-3, (prec, resid)
        assert all(abs(r["courant"] - 0.5) < 1e-6 for r in recs[1:])
        assert all(abs(r["injected_power"] - 0.1) < 1e-12 for r in recs)
        out[prec] = (u.to(torch.complex128).cpu(), np.array([r["dissipation"] for r in recs]), es, resid)
        b.close()
    (u64, d64, e64, r64), (u32, d32, e32, r32) = out["fp64"], out["fp32"]
    dd = float(np.max(np.abs(d32 - d64) / d64))
    live = e64 >= 1e-9 * e64.sum()
    ek = float(np.max(np.abs(e32[live] - e64[live]) / e64[live]))
    ev = float((u32 - u64).abs().norm() / u64.abs().norm())
    print(f"config 1, 500 steps: budget residual fp64 {r64:.2e} fp32 {r32:.2e}; fp32 vs fp64: D {dd:.2e}, "
          f"E(k) {ek:.2e}, velocity {ev:.2e}")
    assert dd < 1e-3 and ek < 1e-2


# ------------------------------------------------------- spherical truncation
@pytest.mark.parametrize("broadband", [False, True])
def test_spherical_truncation(broadband):
    """The spherical option (parameters.f90:48): the right-hand side masks
    |k| >= (N/2) alpha_x / 2 as rhs.f90:74-88 does, state_dealias masks
    |k| >= (N/2)(2/3) alpha_x as state.f90:186-199 does, and fixed-dt Heun steps
    follow the oracle.  A dealiased field steps through the pruned passes, one
    with broadband content through the full passes.  FP64, 1e-12."""
    n, dt, ns = 32, 2e-3, 6
    uh = field(n, seed=21, k0=3.0, nyquist=broadband)
    p = O.Params(nx=n, ny=n, nz=n, nu=0.01, kCutOff=2.5, Pin=0.1, bandlim=True, spherical=True, tstep_fix=True)
    g = O.Grid(p)
    b = box(n, nu=0.01, kCutOff=2.5, Pin=0.1, bandlim=True, spherical=True, tstep_fix=True, dt=dt)
    got, _ = b.rhs_nonlinear(b.from_numpy(uh))
    assert rel(got.cpu().numpy(), O.rhs_nonlinear(g, uh)) < FP64_TOL
    d = b.from_numpy(uh)
    b.dealias(d)
    assert rel(d.cpu().numpy(), O.state_dealias(g, uh)) < FP64_TOL
    want, _ = O.drive(g, uh, ns, dt)
    u = b.from_numpy(uh)
    b.step(u, ns)
    assert b.step_pruned() == (not broadband)
    assert rel(u.cpu().numpy(), want) < FP64_TOL


def test_spherical_truncation_tc_split():
    """Spherical truncation with the tensor-core passes (128^3): one
    right-hand side against the oracle, the FP32 forms' bar 2e-5."""
    n = 128
    uh = ic.random_field(n, seed=22, k0=3.0)
    p = O.Params(nx=n, ny=n, nz=n, nu=0.01, kCutOff=2.5, Pin=0.1, bandlim=True, spherical=True)
    want = O.rhs_nonlinear(O.Grid(p), uh)
    b = box(n, "tc_split", nu=0.01, kCutOff=2.5, Pin=0.1, bandlim=True, spherical=True)
    got, _ = b.rhs_nonlinear(b.from_numpy(uh))
    assert rel(got.cpu().numpy(), want) < FP32_TOL
