"""Run files from a live box: a saved state holds the oracle's physical
velocity (state_uhat2u) and loads back (R2C, dealias, project) to the same
spectral state; Ekin.dat rows and the spectrum file agree with the step
records and the spectrum call."""
import numpy as np
import pytest

from oracle import dnsbox_oracle as O
from dnsbox_b200 import ic
from dnsbox_b200 import runfiles as R

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec, bar", [("fp64", 1e-14), ("fp32", 1e-6)])
def test_state_save_load_round_trip(tmp_path, prec, bar):
    from dnsbox_b200.ops import Box
    n = 32
    b = Box(n, precision=prec, nu=2e-3, kCutOff=2.5, Pin=0.1)
    uh = b.from_numpy(ic.random_field(n, seed=5, k0=3.0))
    path = R.save_state(b, uh, 7, str(tmp_path), time=1.25, step=40)
    assert path.endswith("state0007.bin")
    back, desc = R.load_state(b, path)
    assert desc["time"] == 1.25 and desc["step"] == 40
    rel = float((back - uh).abs().norm() / uh.abs().norm())
    assert rel < bar
    phys, _ = R.read_state_file(path)
    g = O.Grid(O.Params(nx=n, ny=n, nz=n))
    want = O.state_uhat2u(g, uh.cpu().numpy().astype(np.complex128))
    assert np.max(np.abs(phys - want)) <= bar * np.max(np.abs(want))


def test_stats_and_spectrum_files(tmp_path):
    from dnsbox_b200.ops import Box
    n = 32
    b = Box(n, precision="fp64", nu=2e-3, kCutOff=2.5, Pin=0.1, courant_min=0.5, courant_max=0.5)
    u = b.from_numpy(ic.random_field(n, seed=6, k0=3.0))
    recs = b.step(u, 4)
    r = recs[-1]
    row = R.stats_row(b, u, r["t"], r["dt"])
    assert abs(row[1] - r["ekin"]) <= 1e-12 * r["ekin"]
    assert abs(row[2] - r["dissipation"]) <= 1e-12 * r["dissipation"]
    w = R.EkinWriter(tmp_path / "Ekin.dat")
    w.write(row)
    w.write(row)
    back = np.loadtxt(tmp_path / "Ekin.dat")
    assert back.shape == (2, 8) and np.allclose(back[0], row, rtol=1e-11, atol=0)
    path = R.save_spectrum(b, u, 1, str(tmp_path))
    sp = np.loadtxt(path)
    es = b.spectrum(u)[0]
    assert sp.shape == (b.nspec, 2) and np.array_equal(sp[:, 0], np.arange(1, b.nspec + 1, dtype=float))
    assert np.allclose(sp[:, 1], es, rtol=1e-11, atol=1e-300)
