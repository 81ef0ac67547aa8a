"""Run files in the reference driver's formats (no GPU): Fortran edit
descriptors, info.dat written as io.f90:704-731 and read as io.f90:733-773 and
python/analysis.py:12-22 read it, Ekin.dat rows (8e20.12) and spectrum rows
(2e20.12) read back with numpy.loadtxt as analysis.py:24 does, and the raw
state file with its layout descriptor."""
import json
import types

import numpy as np
import pytest

from dnsbox_b200 import runfiles as R


@pytest.mark.parametrize("x, want", [
    (1.0, "  0.100000000000E+01"),
    (0.0, "  0.000000000000E+00"),
    (-2.5e-7, " -0.250000000000E-06"),
    (123.456, "  0.123456000000E+03"),
    (0.9999999999999, "  0.100000000000E+01"),      # rounds up into the next decade
    (1e100, "  0.100000000000+101"),                 # three-digit exponent drops the E
    (-3.0e-120, " -0.300000000000-119"),
    (0.5, "  0.500000000000E+00"),
])
def test_fortran_e20_12(x, want):
    got = R.fortran_e(x)
    assert got == want and len(got) == 20


def test_fortran_f_and_i():
    assert R.fortran_f(1.0, 12, 9) == " 1.000000000"
    assert R.fortran_f(0.002, 12, 9) == " 0.002000000"
    assert R.fortran_f(-0.5, 12, 9) == "-0.500000000"
    assert R.fortran_f(1234.5, 12, 9) == "*" * 12          # does not fit F12.9
    assert R.fortran_i(64, 4) == "  64"
    assert R.fortran_i(12345, 4) == "****"


def _fake_box(bandlim):
    p = types.SimpleNamespace(alpha_x=1.0, alpha_y=2.0, alpha_z=0.5, dt=0.001, nu=0.002, bandlim=bandlim,
                              Pin=0.1, kCutOff=2.5, Q=0.25, Deltak=1.0, courant_max=0.5)
    return types.SimpleNamespace(params=p, nx=64, ny=32, nz=128)


@pytest.mark.parametrize("bandlim", [True, False])
def test_info_dat_layout_and_readers(tmp_path, bandlim):
    path = tmp_path / "info.dat"
    R.write_info(path, _fake_box(bandlim), courant=0.5)
    lines = path.read_text().splitlines()
    assert lines[0] == "Nx,y,z =   64  32 128"
    assert lines[1] == "iSaveRate1 =   1000" and lines[2] == "iSaveRate2 =     10"
    assert lines[3] == "alpha_x,y,z =  1.000000000 2.000000000 0.500000000"
    assert lines[4] == "dt =  0.001000000" and lines[5] == "nu =  0.002000000"
    if bandlim:
        assert lines[6] == "Pin =  0.100000000" and lines[7] == "kF =  2.500000000"
    else:
        assert lines[6] == "Q =  0.250000000"
    assert lines[-1] == " Random initial condition"
    # io.f90:733-773
    info = R.read_info(path)
    assert (info["nx"], info["ny"], info["nz"]) == (64, 32, 128) and info["alpha"] == (1.0, 2.0, 0.5)
    # python/analysis.py:12-22 (line 6 is Q, or Pin for a band-forced run)
    for i, line in enumerate(lines):
        if i == 3:
            assert [float(t) for t in line.split()[2:5]] == [1.0, 2.0, 0.5]
        if i == 5:
            assert float(line.split()[2]) == 0.002
        if i == 6:
            assert float(line.split()[2]) == (0.1 if bandlim else 0.25)


def test_ekin_and_spectrum_rows_load_back(tmp_path):
    rng = np.random.default_rng(0)
    rows = rng.standard_normal((5, 8)) * 10.0 ** rng.integers(-8, 8, (5, 8))
    w = R.EkinWriter(tmp_path / "Ekin.dat")
    for r in rows:
        w.write(r)
    text = (tmp_path / "Ekin.dat").read_text().splitlines()
    assert all(len(line) == 160 for line in text)
    back = np.loadtxt(tmp_path / "Ekin.dat")
    assert back.shape == (5, 8)
    assert np.all(np.abs(back - rows) <= 5e-12 * np.abs(rows))   # 12 significant digits
    with pytest.raises(ValueError):
        w.write(rows[0][:7])
    k = np.arange(1, 11, dtype=float)
    e = k ** -5.0 / 3.0
    R.write_spectrum(tmp_path / "spec0001.dat", k, e)
    sp = np.loadtxt(tmp_path / "spec0001.dat")
    assert sp.shape == (10, 2) and np.array_equal(sp[:, 0], k)
    assert np.all(np.abs(sp[:, 1] - e) <= 5e-12 * e)


def test_state_file_reader(tmp_path):
    nx, ny, nz = 8, 6, 4
    u = np.arange(3 * nz * ny * nx, dtype=np.float64).reshape(3, nz, ny, nx) / 7.0
    base = tmp_path / "state0003"
    u.astype("<f8").tofile(str(base) + ".bin")
    desc = {"shape_per_field": [nz, ny, nx], "nx": nx, "ny": ny, "nz": nz}
    (tmp_path / "state0003.json").write_text(json.dumps(desc))
    got, d = R.read_state_file(str(base) + ".bin")
    assert np.array_equal(got, u) and d["nx"] == nx
    # a truncated file is refused
    u[:, :2].astype("<f8").tofile(str(base) + ".bin")
    with pytest.raises(ValueError):
        R.read_state_file(str(base) + ".bin")


def test_batched_box_is_refused():
    box = types.SimpleNamespace(nbatch=4, nx=8, ny=8, nz=8, params=_fake_box(True).params)
    for fn in (lambda: R.stats_row(box, None, 0.0, 1e-3), lambda: R.save_spectrum(box, None, 1),
               lambda: R.save_state(box, None, 1), lambda: R.load_state(box, "x.bin")):
        with pytest.raises(ValueError):
            fn()
