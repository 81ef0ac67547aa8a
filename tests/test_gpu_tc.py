"""Tensor-core split-precision form (precision "tc_split") on the GPU.

The strided (y and z) transforms of lengths 128 .. 1024 run their 64-point
first stage as tcgen05 MMAs on hi + lo f16 splits of per-pencil scaled FP32
data (FP32 accumulation in tensor memory); the x axis, the fused z finish and
axes of other lengths use the FP32 kernels, and the state is FP32.

Bars: transforms and one right-hand side against the FP64 oracle within
single-precision tolerances; trajectories against the plain FP64 GPU form for
the velocity (relative L2), the E(k) shells and the dissipation, with the
tolerance written beside each case."""
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


def box(precision="tc_split", n=None, **kw):
    from dnsbox_b200.ops import Box
    return Box(n, precision=precision, **kw)


@pytest.mark.parametrize("shape", [(128, 128, 128), (64, 256, 128), (96, 128, 512), (16, 1024, 256)])
def test_tc_transforms_match_pocketfft(shape):
    nx, ny, nz = shape
    b = box(nx=nx, ny=ny, nz=nz)
    g = O.Grid(O.Params(nx=nx, ny=ny, nz=nz))
    rng = np.random.default_rng(7)
    f = rng.standard_normal((nz, ny, nx))
    F = g.r2c(f)
    Fg = b.r2c(torch.from_numpy(f).to(b.device, b.rdtype)).cpu().numpy()
    e_r2c = rel(Fg, F)
    fg = b.c2r(torch.from_numpy(F).to(b.device, b.cdtype)).cpu().numpy()
    e_c2r = rel(fg, g.c2r(F))
    print(f"tc transforms {shape}: r2c {e_r2c:.3e} c2r {e_c2r:.3e}")
    assert e_r2c < 8e-7 and e_c2r < 8e-7   # measured 2-3e-7: a few ulp of 2^-24 per pass


def test_tc_path_is_taken_and_close_to_fp32():
    """The TC form differs bitwise from the FP32 kernels (a different DFT
    evaluation) but agrees with them to single-precision accuracy."""
    n = 128
    rng = np.random.default_rng(3)
    f = rng.standard_normal((n, n, n)).astype(np.float32)
    b32, btc = box("fp32", n), box("tc_split", n)
    a = b32.r2c(torch.from_numpy(f).to(b32.device)).cpu().numpy()
    t = btc.r2c(torch.from_numpy(f).to(btc.device)).cpu().numpy()
    assert not np.array_equal(a, t)
    assert rel(t, a) < 1e-6


@pytest.mark.parametrize("e", [-60, 60])
def test_tc_power_of_two_scale_invariance(e):
    """Per-pencil power-of-two scaling makes the split exact under a global
    2^e scale: fields far outside the f16 range (2^-60, 2^60) give the
    unit-scale result times 2^e, bit for bit."""
    n = 128
    rng = np.random.default_rng(5)
    f = torch.from_numpy(rng.standard_normal((n, n, n)).astype(np.float32))
    b = box(n=n)
    one = b.r2c(f.to(b.device))
    scaled = b.r2c((f * 2.0 ** e).to(b.device))
    assert torch.equal(scaled, one * 2.0 ** e)
    back = b.c2r(one * 2.0 ** e)
    assert torch.equal(back, b.c2r(one) * 2.0 ** e)


@pytest.mark.parametrize("n", [128, 256])
def test_tc_rhs_nonlinear(n):
    uh = ic.random_field(n, seed=n + 1, k0=3.0)
    p = O.Params(nx=n, ny=n, nz=n, nu=2e-3, kCutOff=2.5, Pin=0.1, bandlim=True)
    want, eb = O.rhs_nonlinear(O.Grid(p), uh, return_eband=True)
    b = box(n=n, nu=2e-3, kCutOff=2.5, Pin=0.1, bandlim=True)
    got, ebg = b.rhs_nonlinear(b.from_numpy(uh))
    e = rel(got.cpu().numpy(), want)
    print(f"tc rhs {n}: {e:.3e}")
    assert e < 2e-6   # same bar as the FP32 form (measured 5e-7)
    assert abs(ebg - eb) < 1e-6 * eb


def _trajectory(prec, n, uh64, nsteps, **kw):
    b = box(prec, n, **kw)
    u = uh64.to(b.device, b.cdtype).clone()
    recs = b.step(u, nsteps)
    es, *_ = b.spectrum(u)
    out = u.to(torch.complex128)
    b.close()
    return out, recs, es


def _errors(u, recs, es, u64, recs64, es64, floor=1e-9):
    """Velocity relative L2; the largest relative E(k) error over shells
    holding at least `floor` of the energy, and over the shells between 1e-14
    and `floor` (reported only: there the modes are 1e-7 .. 1e-5 of the peak
    amplitude and FP32 storage round-off dominates both FP32 forms; shells
    past the dealiasing cube hold FP64 round-off only); the largest relative
    dissipation error over the steps."""
    ev = float((u - u64).abs().norm() / u64.abs().norm())
    sh = np.abs(es - es64) / np.where(es64 > 0, es64, 1.0)
    tot = es64.sum()
    ek = float(np.max(sh[es64 >= floor * tot]))
    tail = (es64 >= 1e-14 * tot) & (es64 < floor * tot)
    ek_all = float(np.max(sh[tail])) if tail.any() else 0.0
    dd = max(abs(a["dissipation"] - r["dissipation"]) / r["dissipation"] for a, r in zip(recs, recs64))
    return ev, ek, ek_all, dd


def test_tc_heun_trajectory_128():
    """Forced turbulence at 128^3, CFL-controlled Heun, 40 steps against the
    plain FP64 GPU form; the FP32 SIMT form is run beside it for scale."""
    n, ns = 128, 40
    kw = dict(nu=2e-3, kCutOff=2.5, Pin=0.1, courant_min=0.5, courant_max=0.5)
    b64 = box("fp64", n, **kw)
    u0 = b64.from_numpy(ic.random_field(n, seed=4, k0=3.0))
    b64.close()
    u64, r64, e64 = _trajectory("fp64", n, u0, ns, **kw)
    res = {}
    for prec in ("fp32", "tc_split"):
        res[prec] = _errors(*_trajectory(prec, n, u0, ns, **kw), u64, r64, e64)
        print(f"{prec} 128^3 {ns} steps: vel {res[prec][0]:.3e} E(k) {res[prec][1]:.3e} "
              f"(tail shells {res[prec][2]:.3e}) D {res[prec][3]:.3e}")
    ev, ek, ek_tail, dd = res["tc_split"]
    assert ev < 1e-6 and ek < 1e-5 and dd < 1e-6
    # tail shells (1e-14 .. 1e-9 of E): bounded, and no worse than the FP32
    # SIMT form's by more than a small factor
    assert ek_tail < 1e-3 and ek_tail < 8 * res["fp32"][2] + 1e-6
    # no worse than the FP32 SIMT form by more than a small factor
    assert ev < 4 * res["fp32"][0] + 1e-7


def test_tc_batched_matches_single():
    n, ns = 128, 3
    kw = dict(nu=2e-3, kCutOff=2.5, Pin=0.1, tstep_fix=True, dt=2e-3)
    us = [ic.random_field(n, seed=s, k0=3.0) for s in (1, 2)]
    from dnsbox_b200.ops import Box
    # the same kernels on both (a schedule tuned for one shape is cached for it alone)
    bb = Box(n, precision="tc_split", nbatch=2, **kw)
    bb.set_schedule((1, 1, 1), 2, False)
    ub = torch.stack([torch.from_numpy(u) for u in us], dim=1).to(bb.device, bb.cdtype).contiguous()
    bb.step(ub, ns)
    for i, u in enumerate(us):
        b1 = box(n=n, **kw)
        b1.set_schedule((1, 1, 1), 2, False)
        u1 = b1.from_numpy(u)
        b1.step(u1, ns)
        assert torch.equal(ub[:, i], u1)


def test_tc_512_accuracy_against_fp64():
    """512^3 forced turbulence (nu = 8e-4, band forcing eps = 0.1, Courant 0.5),
    100 Heun steps from the seeded k0 = 3 field: TC-split against the plain
    FP64 GPU form.  Bars: velocity relative L2 <= 1e-6; E(k) <= 1e-5 on every
    shell holding at least 1e-9 of the energy and <= 1e-3 on the shells between
    1e-14 and 1e-9 of it (there the FP32 transforms' error, which is relative to
    the whole field, dominates: the FP32 SIMT form measures the same);
    dissipation <= 1e-5 on every step."""
    from dnsbox_b200.ic import random_field_gpu
    n, ns = 512, 100
    kw = dict(nu=8e-4, kCutOff=2.5, Pin=0.1, courant_min=0.5, courant_max=0.5)
    b64 = box("fp64", n, **kw)
    u0 = random_field_gpu(b64, seed=0, k0=3.0)
    b64.close()
    u0h = u0.cpu()
    del u0
    u64, r64, e64 = _trajectory("fp64", n, u0h.cuda(), ns, **kw)
    u64h = u64.cpu()
    del u64
    torch.cuda.empty_cache()
    res = {}
    for prec in ("fp32", "tc_split"):
        u, r, e = _trajectory(prec, n, u0h.cuda(), ns, **kw)
        res[prec] = _errors(u.cpu(), r, e, u64h, r64, e64)
        del u
        torch.cuda.empty_cache()
        print(f"{prec} 512^3 {ns} steps: vel {res[prec][0]:.3e} E(k) {res[prec][1]:.3e} "
              f"(tail shells {res[prec][2]:.3e}) D {res[prec][3]:.3e}")
    ev, ek, ek_tail, dd = res["tc_split"]
    assert ev < 1e-6 and ek < 1e-5 and dd < 1e-5
    # measured: TC-split 6.0e-4, FP32 1.1e-4 on the tail shells
    assert ek_tail < 1e-3 and ek_tail < 8 * res["fp32"][2] + 1e-6


def test_tc_1024_energy_budget():
    """1024^3 forced turbulence in the TC-split form (FP32 state, nu = 4e-4,
    band forcing eps = 0.1, Courant 0.5), 20 Heun steps from the seeded k0 = 3
    field: finite, Courant held at 0.5, and the energy budget
    dE/dt = Pin - D (trapezoidal D) within 1e-3 (1% of Pin) on every step
    (measured 3e-5: the time-stepping error of the budget estimate)."""
    from dnsbox_b200.ic import random_field_gpu
    n, ns = 1024, 20
    b = box(n=n, nu=4e-4, kCutOff=2.5, Pin=0.1, courant_min=0.5, courant_max=0.5)
    u = random_field_gpu(b, seed=0, k0=3.0)
    torch.cuda.empty_cache()
    e0 = b.kinetic(u)
    recs = b.step(u, ns)
    es = [e0] + [r["ekin"] for r in recs]
    worst = 0.0
    for i in range(1, ns):
        dEdt = (es[i + 1] - es[i]) / recs[i]["dt"]
        worst = max(worst, abs(dEdt - (0.1 - 0.5 * (recs[i - 1]["dissipation"] + recs[i]["dissipation"]))))
    print(f"tc_split 1024^3 {ns} steps: E {es[0]:.6f} -> {es[-1]:.6f}, worst budget residual {worst:.2e}, "
          f"Courant {recs[-1]['courant']:.6f}")
    assert all(np.isfinite(r["ekin"]) for r in recs)
    assert all(abs(r["courant"] - 0.5) < 1e-5 for r in recs[1:])
    assert worst < 1e-3
    b.close()
    del u
    torch.cuda.empty_cache()


def test_tc_rhs_anisotropic_box():
    """One right-hand side on an anisotropic box, x 64, y 128, z 256 with
    alpha 1, 2, 0.5: tensor-core passes of two lengths and a 2/3 cut at a
    different index on every axis, against the FP64 oracle (the FP32 form's
    bar, 2e-6)."""
    nx, ny, nz = 64, 128, 256
    alpha = (1.0, 2.0, 0.5)
    p = O.Params(nx=nx, ny=ny, nz=nz, alpha_x=alpha[0], alpha_y=alpha[1], alpha_z=alpha[2], nu=2e-3,
                 kCutOff=2.5, Pin=0.1, bandlim=True)
    g = O.Grid(p)
    rng = np.random.default_rng(11)
    uh = O.state_dealias(g, O.state_project(g, O.state_u2uhat(g, rng.standard_normal((3, nz, ny, nx)))))
    uh = uh * np.sqrt(0.5 / O.state_kinetic(g, uh))
    want, eb = O.rhs_nonlinear(g, uh, return_eband=True)
    b = box(nx=nx, ny=ny, nz=nz, alpha=alpha, nu=2e-3, kCutOff=2.5, Pin=0.1, bandlim=True)
    got, ebg = b.rhs_nonlinear(b.from_numpy(uh))
    e = rel(got.cpu().numpy(), want)
    print(f"tc rhs anisotropic {nx}x{ny}x{nz}: {e:.3e}")
    assert e < 2e-6
    assert abs(ebg - eb) < 1e-6 * eb
    b.close()
