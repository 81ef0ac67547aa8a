"""Pruned passes (2/3-rule zeros) against the full passes: bit-identical states
and step records, for every precision form, both steppers, CFL control,
anisotropic boxes, sizes whose cut falls exactly on a wavenumber (48, 96) and
the sizes that run the tensor-core and warp-granular kernels; and the fallback
to the full passes for a state that does not vanish on the cut set."""
import numpy as np
import pytest
import torch

from oracle import dnsbox_oracle as O
from dnsbox_b200 import ic

pytestmark = pytest.mark.gpu


def dealiased(nx, ny, nz, seed, alpha=(1.0, 1.0, 1.0)):
    g = O.Grid(O.Params(nx=nx, ny=ny, nz=nz, alpha_x=alpha[0], alpha_y=alpha[1], alpha_z=alpha[2]))
    rng = np.random.default_rng(seed)
    u = O.state_dealias(g, O.state_project(g, O.state_u2uhat(g, rng.standard_normal((3, nz, ny, nx)))))
    return u * (0.7 / np.sqrt(O.state_kinetic(g, u)))


def run_pair(shape, prec, nsteps, uh, alpha=(1.0, 1.0, 1.0), **kw):
    from dnsbox_b200.ops import Box
    nx, ny, nz = shape
    out = []
    for prune in (True, False):
        b = Box(nx=nx, ny=ny, nz=nz, precision=prec, alpha=alpha, prune=prune, **kw)
        u = b.from_numpy(uh)
        recs = b.step(u, nsteps)
        out.append((u.cpu(), recs, b.step_pruned()))
        b.close()
    return out


FORCED = dict(nu=2e-3, kCutOff=2.5, Pin=0.1, courant_min=0.5, courant_max=0.5)


@pytest.mark.parametrize("prec", ["fp64", "fp32", "tc_split"])
@pytest.mark.parametrize("shape", [(32, 32, 32), (48, 48, 48), (96, 96, 96), (128, 128, 128), (256, 256, 256),
                                   (64, 32, 128)])
def test_pruned_heun_cfl_bit_identical(prec, shape):
    uh = ic.random_field(shape[0], seed=1, k0=3.0) if len(set(shape)) == 1 else dealiased(*shape, seed=1)
    (up, rp, pr), (uf, rf, pf) = run_pair(shape, prec, 6, uh, **FORCED)
    assert pr and not pf
    assert torch.equal(up, uf)
    for a, b in zip(rp, rf):
        assert (a["ekin"], a["dissipation"], a["dt"], a["courant"]) == (b["ekin"], b["dissipation"], b["dt"],
                                                                        b["courant"])


@pytest.mark.parametrize("prec", ["fp64", "fp32", "tc_split"])
@pytest.mark.parametrize("ab2", ["reference", "standard"])
def test_pruned_ab2_bit_identical(prec, ab2):
    n = 128 if prec == "tc_split" else 64   # the tensor-core passes start at 128
    uh = ic.random_field(n, seed=2, k0=4.0)
    (up, rp, pr), (uf, rf, _) = run_pair((n, n, n), prec, 8, uh, nu=0.01, bandlim=False, stepper="ab2", ab2=ab2,
                                         tstep_fix=True, dt=2e-3)
    assert pr and torch.equal(up, uf)
    assert [r["dissipation"] for r in rp] == [r["dissipation"] for r in rf]


def test_pruned_anisotropic_box():
    shape, alpha = (48, 32, 64), (1.0, 2.0, 0.5)
    uh = dealiased(*shape, seed=3, alpha=alpha)
    (up, _, pr), (uf, _, _) = run_pair(shape, "fp64", 5, uh, alpha=alpha, nu=0.01, kCutOff=3.0, Pin=0.2)
    assert pr and torch.equal(up, uf)


def test_state_with_cut_content_takes_the_full_path():
    """Content on the cut set (here a single mode, and a Nyquist-free broadband
    field) is detected; the call then runs the full passes."""
    n = 32
    uh = ic.random_field(n, seed=4, k0=3.0)
    uh[0, 5, 3, 13] = 1e-3 + 2e-3j          # kx = 13 >= 32/3 (not the Nyquist column 16): cut
    (up, _, pr), (uf, _, _) = run_pair((n, n, n), "fp64", 3, uh, **FORCED)
    assert not pr and torch.equal(up, uf)
