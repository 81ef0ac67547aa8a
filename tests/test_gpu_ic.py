"""Initial conditions on the device (state.f90:211-307) and the band driver's
per-step projection (dnsboxband.f90:142-143) against the oracle."""
import numpy as np
import pytest
import torch

from oracle import dnsbox_oracle as O
from dnsbox_b200 import ic

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("mode", ["mpi", "single"])
def test_yoffe_matches_oracle_with_shared_noise(mode):
    from dnsbox_b200.ops import Box
    n = 32
    g = O.Grid(O.Params(nx=n, ny=n, nz=n, spectrum_mode=mode))
    noise = np.random.default_rng(21).random((3, n, n, n)) - 0.5
    want = O.state_init_rand(g, noise)
    b = Box(n, spectrum_mode=mode)
    got = b.init_yoffe(torch.from_numpy(noise).to(b.device))
    assert rel(got.cpu().numpy(), want) < 1e-12
    b.close()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_yoffe_seeded_has_the_target_spectrum(prec):
    """Drawn on the device: solenoidal, dealiased, and in the spectrum mode it
    was rescaled with every shell 1 .. Nspec-1 holds C1 k^C2 exp(-C3 k^C4)."""
    from dnsbox_b200.ops import Box
    n = 48
    b = Box(n, precision=prec)
    u = b.init_yoffe(seed=7)
    es, *_ = b.spectrum(u)
    c1, c2, c3, c4 = O.YOFFE_C
    k = np.arange(1, b.nspec)
    target = c1 * k ** c2 * np.exp(-c3 * k ** c4)
    tol = 1e-12 if prec == "fp64" else 2e-6
    assert np.max(np.abs(es[: b.nspec - 1] - target) / target) < tol
    assert es[b.nspec - 1] == 0.0
    g = O.Grid(O.Params(nx=n, ny=n, nz=n))
    uh = u.cpu().numpy().astype(np.complex128)
    assert rel(O.state_dealias(g, O.state_project(g, uh)), uh) < (1e-14 if prec == "fp64" else 1e-7)
    b.close()


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 8e-7)])
def test_beltrami_matches_oracle(prec, tol):
    from dnsbox_b200.ops import Box
    n, t = 24, 0.37
    b = Box(n, precision=prec, nu=0.02)
    g = O.Grid(O.Params(nx=n, ny=n, nz=n, nu=0.02))
    got = b.init_beltrami(t)
    assert rel(got.cpu().numpy(), O.state_u2uhat(g, O.beltrami(g, t))) < tol
    b.close()


@pytest.mark.parametrize("prune", [True, False])
def test_step_projection_matches_band_driver(prune):
    """Heun steps each followed by state_project and state_dealias (the band
    driver), FP64, against the oracle, with the step records' kinetic energy
    of the projected state."""
    from dnsbox_b200.ops import Box
    n, dt, ns = 24, 3e-3, 3
    kw = dict(nu=0.01, kCutOff=2.5, Pin=0.1, bandlim=True)
    g = O.Grid(O.Params(nx=n, ny=n, nz=n, **kw))
    uh = ic.random_field(n, seed=9, k0=3.0)
    b = Box(n, tstep_fix=True, dt=dt, prune=prune, **kw)
    b.set_step_projection(True)
    u = b.from_numpy(uh)
    recs = b.step(u, ns)
    want = uh
    for r in recs:
        want = O.state_dealias(g, O.state_project(g, O.heun_step(g, want, dt)))
    assert rel(u.cpu().numpy(), want) < 1e-12
    assert abs(recs[-1]["ekin"] - O.state_kinetic(g, want)) < 1e-12 * O.state_kinetic(g, want)
    b.close()
