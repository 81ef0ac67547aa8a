"""Generate golden vectors by running the reference's NumPy prototype.

The reference prototype ``python/dnsbox.py`` is Python 2 code that imports
pylab; its source is executed UNMODIFIED here under a small compatibility
shim: integer-casting ``range`` (Python 2 integer division of ``Nx / 2``), an
empty ``pylab`` module and an ``open`` that captures the stats line instead
of writing a file.  Its functions then produce, on seeded fields:

* ``nonLinear`` (python/dnsbox.py:354-404): the rotational-form nonlinear term
  with the dealias mask set to the Fortran one (rhs.f90:74-88) -- unforced,
  and band forced (the prototype adds the forcing term to every mode, so only
  the forcing coefficient Pin/(2 Eband) is compared from that run);
* ``timeStep`` (python/dnsbox.py:407-442): three IF Heun steps at fixed dt;
* ``stats`` (python/dnsbox.py:486-517): kinetic energy, dissipation, Courant
  number and maximum divergence;
* the Beltrami analytic run of ``init(analytic=True)``.

Outputs are stored as half spectra in the [kz, ky, kx] layout.  Run in this
container only (it reads the reference tree); the .npz files are committed.

    python tests/golden/make_golden.py /root/reference/python/dnsbox.py
"""
from __future__ import annotations

import builtins
import io
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from dnsbox_b200 import ic  # noqa: E402


class _Capture(io.StringIO):
    lines: list = []

    def close(self):
        _Capture.lines.append(self.getvalue())
        super().close()


def _load_prototype(path):
    src = open(path).read()
    sys.modules["pylab"] = types.ModuleType("pylab")
    ns = {
        "__name__": "dnsbox_prototype",
        "range": lambda *a: builtins.range(*[int(x) for x in a]),
        "open": lambda *a, **k: _Capture(),
        "loglog": lambda *a, **k: None,
        "show": lambda *a, **k: None,
    }
    exec(compile(src, path, "exec"), ns)
    return ns


def _full_from_half(uh, n):
    """Hermitian extension of a [kz, ky, kx] half spectrum to the prototype's
    full [x, y, z] spectrum (index [kx, ky, kz])."""
    import scipy.fft as sfft
    phys = sfft.irfftn(uh, s=(n, n, n), axes=(-3, -2, -1))
    full = sfft.fftn(phys, axes=(-3, -2, -1))          # [kz, ky, kx]
    return np.transpose(full, (0, 3, 2, 1)) if full.ndim == 4 else full.T


def _half_from_full(F, n):
    """[kx, ky, kz] full spectrum -> [kz, ky, kx] half spectrum."""
    return np.ascontiguousarray(np.transpose(F, (2, 1, 0))[:, :, : n // 2 + 1])


def _fortran_masks(ns, n, kcut):
    kxm = np.real(ns["kxm"])
    kym = np.real(ns["kym"])
    kzm = np.real(ns["kzm"])
    c = (n / 2.0) * (2.0 / 3.0)
    dealias = np.ones((n, n, n))
    dealias[(np.abs(kxm) >= c) | (np.abs(kym) >= c) | (np.abs(kzm) >= c)] = 0.0
    dealias[(kxm == 0) & (kym == 0) & (kzm == 0)] = 0.0
    kk = kxm ** 2 + kym ** 2 + kzm ** 2
    force = np.where(np.sqrt(kk) <= kcut, 1.0, 0.0)
    return dealias, force


def make(path, n, seed, out):
    ns = _load_prototype(path)
    nu, dt, kcut, pin = 0.01, 2.0e-3, 2.5, 0.1
    ns.update(Nx=n, Ny=n, Nz=n, nu=nu, Q=0.0, analytic=True, random=False,
              tStepFix=True, tStepMax=dt, bandlim=False, kF=kcut, epsW=pin,
              spherical=False)
    ns["init"]()                                   # grids, kxm.., Beltrami state
    dealias, force = _fortran_masks(ns, n, kcut)
    ns["dealias"] = dealias
    ns["force"] = force

    # Beltrami known-answer run: 3 Heun steps from the analytic field
    ns["uhat"] = dealias * ns["uhat"]
    ns["vhat"] = dealias * ns["vhat"]
    ns["what"] = dealias * ns["what"]
    bel0 = np.stack([_half_from_full(ns[c], n) for c in ("uhat", "vhat", "what")])
    ns["uhattemp"], ns["vhattemp"], ns["whattemp"] = (
        ns["uhat"].copy(), ns["vhat"].copy(), ns["what"].copy())
    ns["t"] = 0.0
    ns["timeStep"](3)
    bel3 = np.stack([_half_from_full(ns[c], n) for c in ("uhat", "vhat", "what")])

    # seeded turbulent field
    uh = ic.random_field(n, seed=seed, k0=3.0)
    full = [_full_from_half(uh[c], n) for c in range(3)]
    ns["uhattemp"], ns["vhattemp"], ns["whattemp"] = [f.copy() for f in full]
    ns["bandlim"] = False
    ns["nonLinear"]()
    n_unforced = np.stack([_half_from_full(ns[c], n)
                           for c in ("nonlinuhat", "nonlinvhat", "nonlinwhat")])
    ns["uhattemp"], ns["vhattemp"], ns["whattemp"] = [f.copy() for f in full]
    ns["bandlim"] = True
    ns["nonLinear"]()
    n_forced = np.stack([_half_from_full(ns[c], n)
                         for c in ("nonlinuhat", "nonlinvhat", "nonlinwhat")])
    ns["bandlim"] = False

    # three Heun steps of the seeded field, then stats
    ns["uhat"], ns["vhat"], ns["what"] = [f.copy() for f in full]
    ns["uhattemp"], ns["vhattemp"], ns["whattemp"] = [f.copy() for f in full]
    ns["t"] = 0.0
    ns["timeStep"](3)
    heun3 = np.stack([_half_from_full(ns[c], n) for c in ("uhat", "vhat", "what")])
    _Capture.lines.clear()
    ns["stats"]()
    vals = [float(x) for x in _Capture.lines[-1].split()]
    t, ek, disp, prod, courant, div = vals
    np.savez_compressed(
        out, n=n, seed=seed, nu=nu, dt=dt, kcut=kcut, pin=pin,
        uh0=uh, n_unforced=n_unforced, n_forced=n_forced, heun3=heun3,
        beltrami0=bel0, beltrami3=bel3,
        stats=np.array([t, ek, disp, prod, courant, div]))
    print(out, "stats", vals)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path to the reference's python/dnsbox.py>")
    proto = sys.argv[1]
    make(proto, 16, 7, os.path.join(HERE, "golden_n16.npz"))
    make(proto, 12, 11, os.path.join(HERE, "golden_n12.npz"))
