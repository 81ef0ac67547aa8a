"""Run files of the reference driver, for resume and for its post-processing.

- ``info.dat``: the run parameters as io.f90:704-731 writes them (Fortran edit
  descriptors I4, I6, F12.9 and one list-directed line), read back the way
  io.f90:733-773 does (list-directed: blanks and commas separate items).
- ``Ekin.dat``: one row of eight E20.12 numbers per save (io.f90:628-661):
  time, kinetic energy, dissipation, input 2QE, Courant number, maximum
  divergence, energy at k = 0, band energy.
- ``specNNNN.dat``: the shell spectrum, rows of two E20.12 numbers
  (kSpec(i) = i Deltak, E(k)), io.f90:680-702.
- the state: the reference writes HDF5 datasets ``u``, ``v``, ``w`` of
  (Nx, Ny, Nz) physical doubles (io.f90:100-278) and loads them back with
  R2C, dealias and projection (dnsboxheun.f90:48-55).  HDF5 is not available
  here, so the same three arrays go to ``stateNNNN.bin`` (FP64, x fastest,
  then y, then z; u, v, w one after another) with a JSON layout descriptor
  ``stateNNNN.json`` beside it.

Everything here is host code; a save moves the physical fields across PCIe
once.  The physical velocity is u = C2R(uhat) / (Nx Ny Nz) and the state is
uhat = R2C(u) (state.f90:74-96).
"""
from __future__ import annotations

import json
import math
import os
import re

import numpy as np

__all__ = ["fortran_e", "fortran_f", "fortran_i", "write_info", "read_info", "EkinWriter", "stats_row",
           "write_spectrum", "save_spectrum", "save_state", "load_state", "read_state_file"]


# ------------------------------------------------------------ edit descriptors
def fortran_e(x: float, w: int = 20, d: int = 12) -> str:
    """Fortran ``Ew.d`` output: [-]0.<d digits>E+ee right-justified in w
    characters (mantissa in [0.1, 1), correctly rounded); exponents beyond
    +-99 take the form +eee without the letter E; w stars if it does not fit."""
    if math.isnan(x):
        return "NaN".rjust(w)
    if math.isinf(x):
        return ("-Infinity" if x < 0 else "Infinity").rjust(w)
    if x == 0.0:
        body = "0." + "0" * d + "E+00"
        s = ("-" if math.copysign(1.0, x) < 0 else "") + body
    else:
        m = f"{abs(x):.{d - 1}e}"   # d significant digits: D.DDDDe+XX, correctly rounded
        digits = m[0] + m[2:2 + d - 1]
        e = int(m[m.index("e") + 1:]) + 1
        exp = f"E{'+' if e >= 0 else '-'}{abs(e):02d}" if abs(e) <= 99 else f"{'+' if e >= 0 else '-'}{abs(e):03d}"
        s = ("-" if x < 0 else "") + "0." + digits + exp
    return s.rjust(w) if len(s) <= w else "*" * w


def fortran_f(x: float, w: int, d: int) -> str:
    """Fortran ``Fw.d`` output (w stars when the value does not fit)."""
    s = f"{x:{w}.{d}f}"
    return s if len(s) <= w else "*" * w


def fortran_i(n: int, w: int) -> str:
    """Fortran ``Iw`` output (w stars when the value does not fit)."""
    s = f"{int(n):{w}d}"
    return s if len(s) <= w else "*" * w


def _single(box):
    if getattr(box, "nbatch", 1) > 1:
        raise ValueError("run files describe one box; take the box out of the batch first")


# ------------------------------------------------------------------ info.dat
def write_info(path, box, *, courant=None, isave1=1000, isave2=10, initrand=True, mode="a"):
    """Append the run parameters of ``box`` to ``path`` in the layout of
    io.f90:704-731 (the reference opens info.dat with access='append')."""
    p = box.params
    lines = [
        "Nx,y,z = " + "".join(fortran_i(v, 4) for v in (box.nx, box.ny, box.nz)),
        "iSaveRate1 = " + fortran_i(isave1, 6),
        "iSaveRate2 = " + fortran_i(isave2, 6),
        "alpha_x,y,z = " + "".join(fortran_f(v, 12, 9) for v in (p.alpha_x, p.alpha_y, p.alpha_z)),
        "dt = " + fortran_f(p.dt, 12, 9),
        "nu = " + fortran_f(p.nu, 12, 9),
    ]
    if p.bandlim:
        lines += ["Pin = " + fortran_f(p.Pin, 12, 9), "kF = " + fortran_f(p.kCutOff, 12, 9)]
    else:
        lines += ["Q = " + fortran_f(p.Q, 12, 9)]
    lines += ["Deltak = " + fortran_f(p.Deltak, 12, 9),
              "Courant = " + fortran_f(p.courant_max if courant is None else courant, 12, 9),
              # list-directed output of a character constant starts with a blank
              " Random initial condition" if initrand else " Initial condition read from file"]
    with open(path, mode) as f:
        f.write("\n".join(lines) + "\n")


_LIST_SEP = re.compile(r"[,\s]+")


def _items(line):
    return [t for t in _LIST_SEP.split(line.strip()) if t]


def read_info(path):
    """The grid and the box lengths' alphas as io.f90:733-773 reads them
    (list-directed: four words, then three values, on lines 1 and 4)."""
    with open(path) as f:
        lines = f.read().splitlines()
    a = _items(lines[0])
    b = _items(lines[3])
    return {"nx": int(a[4]), "ny": int(a[5]), "nz": int(a[6]),
            "alpha": (float(b[4]), float(b[5]), float(b[6]))}


# ------------------------------------------------------------------ Ekin.dat
def stats_row(box, uh, t, dt):
    """The eight Ekin.dat quantities at state ``uh`` and time t (io.f90:628-661):
    time, Ekin, dissipation, input 2 Q Ekin, Courant number at step dt,
    maximum divergence, EZero (state_spectrum), Eband (rhs_Eband)."""
    _single(box)
    ekin = box.kinetic(uh)
    disp = box.dissipation(uh)
    courant, _ = box.courant(uh, dt)
    div = box.divergence(uh)
    _, ezero, _, _ = box.spectrum(uh)
    eband = box.eband(uh) if box.params.bandlim else 0.0
    return (float(t), ekin, disp, 2.0 * box.params.Q * ekin, courant, div, ezero, eband)


class EkinWriter:
    """Appends Ekin.dat rows (format 8e20.12)."""

    def __init__(self, path):
        self.path = path

    def write(self, row):
        if len(row) != 8:
            raise ValueError("an Ekin.dat row has 8 columns")
        with open(self.path, "a") as f:
            f.write("".join(fortran_e(float(v)) for v in row) + "\n")


# ---------------------------------------------------------------- spectrum
def write_spectrum(path, kspec, espec):
    """Appends rows (k, E(k)) in format 2e20.12 (io.f90:680-702)."""
    with open(path, "a") as f:
        for k, e in zip(kspec, espec):
            f.write(fortran_e(float(k)) + fortran_e(float(e)) + "\n")


def save_spectrum(box, uh, count, directory="."):
    """state_spectrum of ``uh`` to specNNNN.dat (NNNN = count, I4.4)."""
    _single(box)
    es, _, _, _ = box.spectrum(uh)
    kspec = (np.arange(1, len(es) + 1) * box.params.Deltak).tolist()
    path = os.path.join(directory, f"spec{count:04d}.dat")
    write_spectrum(path, kspec, es)
    return path


# ------------------------------------------------------------------- state
def save_state(box, uh, count, directory=".", time=0.0, step=0):
    """Physical u, v, w (FP64) of the spectral state ``uh`` to stateNNNN.bin
    plus the layout descriptor stateNNNN.json; returns the .bin path."""
    import torch
    _single(box)
    s = 1.0 / (box.nx * box.ny * box.nz)
    base = os.path.join(directory, f"state{count:04d}")
    with open(base + ".bin", "wb") as f:
        for c in range(3):
            phys = (box.c2r(uh[c].contiguous()) * s).to(torch.float64).cpu().numpy()
            f.write(np.ascontiguousarray(phys).tobytes())
    p = box.params
    desc = {"format": "dnsbox state, raw float64", "fields": ["u", "v", "w"],
            "shape_per_field": [box.nz, box.ny, box.nx], "order": "x fastest, then y, then z",
            "nx": box.nx, "ny": box.ny, "nz": box.nz, "alpha": [p.alpha_x, p.alpha_y, p.alpha_z],
            "time": float(time), "step": int(step), "byteorder": "little"}
    with open(base + ".json", "w") as f:
        json.dump(desc, f, indent=1)
    return base + ".bin"


def read_state_file(path):
    """(u, v, w) physical fields (3, nz, ny, nx) FP64 and the descriptor."""
    base = path[:-4] if path.endswith(".bin") else path
    with open(base + ".json") as f:
        desc = json.load(f)
    nz, ny, nx = desc["shape_per_field"]
    a = np.fromfile(base + ".bin", dtype="<f8")
    if a.size != 3 * nx * ny * nz:
        raise ValueError(f"{base}.bin holds {a.size} doubles, the descriptor says {3 * nx * ny * nz}")
    return a.reshape(3, nz, ny, nx), desc


def load_state(box, path):
    """A state file to the spectral state of ``box``: R2C of the physical
    fields, then dealias and projection (dnsboxheun.f90:48-55)."""
    import torch
    _single(box)
    phys, desc = read_state_file(path)
    if (desc["nx"], desc["ny"], desc["nz"]) != (box.nx, box.ny, box.nz):
        raise ValueError(f"state is {desc['nx']}x{desc['ny']}x{desc['nz']}, the box "
                         f"{box.nx}x{box.ny}x{box.nz}")
    uh = box.zeros()
    for c in range(3):
        uh[c] = box.r2c(torch.from_numpy(phys[c]).to(box.device, box.rdtype))
    box.dealias(uh)
    box.project(uh)
    return uh, desc
