"""Host-side grid constants of the dnsbox box (wavenumber tables, shell count).

These mirror ``var_init`` (variables.f90:99-280): wavenumbers are integer
multiples of alpha with the Nyquist entry set to zero in every direction
(variables.f90:229,245,259), ``scalemodes = 1/(Nx Ny Nz)`` (variables.f90:273)
and ``Nspec`` from the cubic (or spherical) truncation radius
(variables.f90:112-123).  The device computes the same tables on the fly from
the mode indices; this module serves host-side set-up (initial conditions,
shell bookkeeping) and the Python API.
"""
from __future__ import annotations

import numpy as np


def k_table(n: int, alpha: float = 1.0, half: bool = False) -> np.ndarray:
    """Real wavenumber of each index along one axis (Nyquist -> 0)."""
    if half:
        k = np.arange(n // 2 + 1, dtype=np.float64) * alpha
        k[n // 2] = 0.0
        return k
    idx = np.arange(n)
    k = np.where(idx < n // 2, idx, idx - n).astype(np.float64) * alpha
    k[n // 2] = 0.0
    return k


def nspec(nx: int, ny: int, nz: int, alpha=(1.0, 1.0, 1.0), deltak: float = 1.0,
          spherical: bool = False) -> int:
    """Number of spectrum shells (variables.f90:112-123)."""
    ax, ay, az = alpha
    if spherical:
        return int(((nx / 2.0) * (2.0 * ax / 3.0)) / deltak) - 1
    return int(np.sqrt(((nx / 2.0) * (2.0 * ax / 3.0)) ** 2
                       + ((ny / 2.0) * (2.0 * ay / 3.0)) ** 2
                       + ((nz / 2.0) * (2.0 * az / 3.0)) ** 2) / deltak) - 1


def spectral_shape(nx: int, ny: int, nz: int):
    """Shape of one spectral field in HBM: [kz][ky][kx], kx fastest, kx <= nx/2."""
    return (nz, ny, nx // 2 + 1)


def physical_shape(nx: int, ny: int, nz: int):
    """Shape of one physical field in HBM: [z][y][x], x fastest."""
    return (nz, ny, nx)


def broadcast_k(nx: int, ny: int, nz: int, alpha=(1.0, 1.0, 1.0)):
    """(kz, ky, kx) real wavenumber arrays broadcastable to the spectral shape."""
    kx = k_table(nx, alpha[0], half=True)[None, None, :]
    ky = k_table(ny, alpha[1])[None, :, None]
    kz = k_table(nz, alpha[2])[:, None, None]
    return kz, ky, kx
