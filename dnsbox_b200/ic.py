"""Seeded initial conditions for the benchmark and parity workloads (host side).

``random_field`` builds the spectral velocity the workloads start from:

1. a real white-noise velocity drawn from NumPy ``PCG64(seed)`` and transformed
   with an unnormalised R2C, so the half spectrum is a complex Gaussian with
   uniform phases and exact Hermitian symmetry on the kx = 0 plane;
2. the Nyquist index planes and the mean mode are zeroed, the 2/3 rule of
   ``state_dealias`` (state.f90:181-209) is applied and the field is Leray
   projected (state.f90:120-179), so it is real, solenoidal and dealiased;
3. every integer shell n (nearest-window rule of state.f90:363-367) is
   rescaled to E(n) = A n^4 exp(-2 n^2 / k0^2), the Rosales-Meneveau form of
   the reference prototype (python/dnsbox.py:258-281), with A set so the
   total kinetic energy (state.f90:429-454 weighting) equals ``energy``.

``beltrami`` returns the analytic Beltrami flow of state.f90:287-307, the
reference's known-answer initial condition.
"""
from __future__ import annotations

import numpy as np
import scipy.fft as sfft

from .grid import broadcast_k


def _workers():
    import os
    return os.cpu_count() or 1


def _kinetic_weight(nxh: int):
    w = np.ones(nxh)
    w[0] = 0.5
    w[nxh - 1] = 0.5          # Nyquist kx index carries kx = 0 (quirk Q1)
    return w[None, None, :]


def random_field(n: int, seed: int = 0, k0: float = 4.0, energy: float = 0.5,
                 alpha=(1.0, 1.0, 1.0), deltak: float = 1.0) -> np.ndarray:
    """Spectral velocity (3, n, n, n//2+1) complex128, unnormalised (uhat = R2C(u))."""
    nx = ny = nz = n
    rng = np.random.Generator(np.random.PCG64(seed))
    u = rng.standard_normal((3, nz, ny, nx))
    uh = sfft.rfftn(u, axes=(-3, -2, -1), workers=_workers())
    del u
    kz, ky, kx = broadcast_k(nx, ny, nz, alpha)
    # Nyquist index planes and the mean mode
    uh[:, :, :, nx // 2] = 0.0
    uh[:, :, ny // 2, :] = 0.0
    uh[:, nz // 2, :, :] = 0.0
    uh[:, 0, 0, 0] = 0.0
    # 2/3 rule (state.f90:191-196)
    cut = (np.abs(kx) >= (nx / 2.0) * (2.0 * alpha[0] / 3.0)) \
        | (np.abs(ky) >= (ny / 2.0) * (2.0 * alpha[1] / 3.0)) \
        | (np.abs(kz) >= (nz / 2.0) * (2.0 * alpha[2] / 3.0))
    cut = np.broadcast_to(cut, uh.shape[1:])
    uh[:, cut] = 0.0
    # Leray projection
    kk = kx * kx + ky * ky + kz * kz
    kk = np.where(kk == 0.0, 1.0, kk)
    kdotu = (kx * uh[0] + ky * uh[1] + kz * uh[2]) / kk
    uh[0] -= kx * kdotu
    uh[1] -= ky * kdotu
    uh[2] -= kz * kdotu
    del kdotu
    # shell rescale to A k^4 exp(-2 k^2 / k0^2)
    absk = np.sqrt(kx * kx + ky * ky + kz * kz)
    absk = np.broadcast_to(absk, uh.shape[1:])
    base = np.floor(absk / deltak)
    nk = np.where(absk < base + 0.5 * deltak, base, base + 1).astype(np.int64)
    s2 = (1.0 / float(nx * ny * nz)) ** 2
    w = _kinetic_weight(nx // 2 + 1)
    e2 = (np.abs(uh[0]) ** 2 + np.abs(uh[1]) ** 2 + np.abs(uh[2]) ** 2) * w * s2
    nmax = int(nk.max()) + 1
    ecur = np.bincount(nk.ravel(), weights=e2.ravel(), minlength=nmax)
    shells = np.arange(nmax, dtype=np.float64) * deltak
    etgt = shells ** 4 * np.exp(-2.0 * shells ** 2 / (k0 * k0))
    fac = np.zeros(nmax)
    ok = (ecur > 0) & (np.arange(nmax) > 0)
    fac[ok] = np.sqrt(etgt[ok] / ecur[ok])
    uh *= fac[nk][None]
    e = float(np.sum((np.abs(uh[0]) ** 2 + np.abs(uh[1]) ** 2 + np.abs(uh[2]) ** 2) * w) * s2)
    uh *= np.sqrt(energy / e)
    return uh


def beltrami(n: int, nu: float, t: float = 0.0, alpha=(1.0, 1.0, 1.0)) -> np.ndarray:
    """Physical Beltrami velocity (3, n, n, n) on the reference grid x_i = i L/N,
    i = -N/2 .. N/2-1 (variables.f90:235-266), state.f90:287-307."""
    L = [2 * np.pi / a for a in alpha]
    x = np.array([i * L[0] / n for i in range(-n // 2, n // 2)])
    y = np.array([i * L[1] / n for i in range(-n // 2, n // 2)])
    z = np.array([i * L[2] / n for i in range(-n // 2, n // 2)])
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    f = np.sqrt(3.0)
    dec = np.exp(-(f ** 2) * t * nu)
    u = -0.5 * (f * np.cos(X) * np.sin(Y) * np.sin(Z) + np.sin(X) * np.cos(Y) * np.cos(Z)) * dec
    v = 0.5 * (f * np.sin(X) * np.cos(Y) * np.sin(Z) - np.cos(X) * np.sin(Y) * np.cos(Z)) * dec
    w = 1.0 * np.cos(X) * np.cos(Y) * np.sin(Z) * dec
    return np.stack([u, v, w])


def to_spectral(u: np.ndarray) -> np.ndarray:
    """Unnormalised R2C of a physical vector field (3, nz, ny, nx)."""
    return sfft.rfftn(u, axes=(-3, -2, -1), workers=_workers())


def kolmogorov_forcing(n: int, amplitude: float = 1.0, kf: int = 4) -> np.ndarray:
    """Spectral Kolmogorov forcing f = (F sin(kf y), 0, 0) on the reference grid
    (unnormalised R2C, (3, n, n, n//2+1)); nonzero only at (kx, ky, kz) = (0, +-kf, 0)."""
    L = 2 * np.pi
    y = np.array([i * L / n for i in range(-n // 2, n // 2)])
    f = np.zeros((3, n, n, n))
    f[0] = amplitude * np.sin(kf * y)[None, :, None]
    return to_spectral(f)


def random_field_gpu(box, seed: int = 0, k0: float = 4.0, energy: float = 0.5):
    """Device-side counterpart of ``random_field`` for large grids: white noise
    from torch's counter-based generator on the device, the library's R2C,
    Nyquist planes and mean mode zeroed, ``dealias`` + ``project`` and the same
    shell rescale to A k^4 exp(-2 k^2/k0^2) with total energy ``energy``.
    Returns a state tensor of the Box's precision (cubic grids)."""
    import torch
    n = box.nx
    gen = torch.Generator(device=box.device).manual_seed(int(seed))
    uh = box.zeros()
    for c in range(3):
        phys = torch.randn((n, n, n), generator=gen, device=box.device, dtype=box.rdtype)
        uh[c] = box.r2c(phys)
        del phys
    uh[:, :, :, n // 2] = 0
    uh[:, :, n // 2, :] = 0
    uh[:, n // 2, :, :] = 0
    uh[:, 0, 0, 0] = 0
    box.dealias(uh)
    box.project(uh)
    kz, ky, kx = [torch.from_numpy(np.ascontiguousarray(k)).to(box.device) for k in broadcast_k(n, n, n)]
    absk = torch.sqrt(kx * kx + ky * ky + kz * kz).expand(n, n, n // 2 + 1)
    base = torch.floor(absk)
    nk = torch.where(absk < base + 0.5, base, base + 1).to(torch.int64)
    w = torch.ones(n // 2 + 1, dtype=torch.float64, device=box.device)
    w[0] = 0.5
    w[n // 2] = 0.5
    s2 = (1.0 / float(n) ** 3) ** 2
    e2 = (uh.abs().to(torch.float64) ** 2).sum(0) * w * s2
    nmax = int(nk.max().item()) + 1
    ecur = torch.bincount(nk.reshape(-1), weights=e2.reshape(-1), minlength=nmax)
    shells = torch.arange(nmax, dtype=torch.float64, device=box.device)
    etgt = shells ** 4 * torch.exp(-2.0 * shells ** 2 / (k0 * k0))
    fac = torch.where((ecur > 0) & (shells > 0), torch.sqrt(etgt / torch.clamp(ecur, min=1e-300)),
                      torch.zeros_like(ecur))
    uh *= fac[nk].to(box.rdtype)
    e = box.kinetic(uh)
    uh *= float(np.sqrt(energy / e))
    return uh
