"""NumPy FP64 restatement of the dnsbox hot path -- TEST INFRASTRUCTURE ONLY.

Layouts (the same as the GPU product, which keeps them in HBM):
  physical field  f[z, y, x]          real, x fastest (the reference's (x, y, z)
                                      Fortran order, variables.f90:171-192)
  spectral field  F[kz, ky, kx]       complex, kx fastest, kx in [0, nx/2]
                                      (a half spectrum; the reference stores the
                                      transpose, p3dfft STRIDE1 (kz, ky, kx) with
                                      kz fastest, variables.f90:193-213)
  vector fields   stacked on a leading axis of length 3 (u, v, w)

Transforms are unnormalised in both directions, as p3dfft's ``ftran_r2c`` /
``btran_c2r`` (state.f90:58-72); code multiplies by ``scalemodes = 1/N^3``
where the reference does (variables.f90:273).  Wavenumbers are purely
imaginary with the Nyquist entry set to zero in every direction
(variables.f90:226-262, quirk Q1).

Every function cites the reference lines it restates.  Quirks:
  Q1 Nyquist wavenumbers are 0 (kept).
  Q2 AB2 old-term coefficient 0.5*(t_n - dt - t_{n-1}) (``ab2="reference"``)
     versus the standard variable-step IF-AB2 (``ab2="standard"``).
  Q3 dealias threshold ``.ge.`` in rhs.f90/state.f90, ``.gt.`` in rhsAdj.f90.
  Q4 state.f90 spectrum (no kx=0 half weight, ``nk >= Nspec`` excluded, the
     Esqrt2 test matches every |k| < sqrt(2)) versus single/state.f90's
     weighted spectrum (``spectrum_mode="single"``).
  Q5 Courant from the current physical velocity (the reference uses a stale
     copy refreshed every iSaveRate1 steps).
  Q6 rhsAdj.f90 subtracts k*phatadj with phatadj never assigned:
     ``adj_phat="intent"`` uses phat, ``adj_phat="literal"`` uses 0.
  Q8 rhsAdj.f90 passes uhattemp straight to p3dfft_btran_c2r, which p3dfft
     (overwrite=.true., variables.f90:154) may destroy; the restatement keeps
     the evident intent (input preserved).
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np
import scipy.fft as sfft

WORKERS = os.cpu_count() or 1


@dataclasses.dataclass
class Params:
    """Runtime form of parameters.f90:11-50 (compile-time there)."""
    nx: int = 64
    ny: int = 64
    nz: int = 64
    alpha_x: float = 1.0
    alpha_y: float = 1.0
    alpha_z: float = 1.0
    nu: float = 0.005
    Q: float = 0.0
    kCutOff: float = 2.0
    Pin: float = 0.1
    Deltak: float = 1.0
    courant_min: float = 0.15
    courant_max: float = 0.2
    dt_max: float = 1.0e-2
    tstep_fix: bool = False
    hminone: bool = True
    spherical: bool = False
    bandlim: bool = True
    ab2: str = "reference"          # Q2
    adj_phat: str = "intent"        # Q6
    spectrum_mode: str = "mpi"      # Q4


class Grid:
    """Wavenumber tables and grid constants of ``var_init`` (variables.f90:99-280)."""

    def __init__(self, p: Params):
        self.p = p
        nx, ny, nz = p.nx, p.ny, p.nz
        self.nxh = nx // 2 + 1
        # variables.f90:226-233: kx(i) = i*(i-1)*alpha_x, kx(1+Nx/2) = 0
        kxr = np.array([i * p.alpha_x for i in range(nx // 2)] + [0.0])
        # variables.f90:242-262: ky, kz full length with negative half and Nyquist = 0
        def full(n, a):
            k = np.zeros(n)
            for i in range(n // 2):
                k[i] = i * a
            k[n // 2] = 0.0
            for i in range(1, n // 2):
                k[i + n // 2] = -k[n // 2 - i]
            return k
        kyr = full(ny, p.alpha_y)
        kzr = full(nz, p.alpha_z)
        self.kxr, self.kyr, self.kzr = kxr, kyr, kzr
        # imaginary wavenumbers broadcast onto the [kz, ky, kx] layout
        self.kx = (1j * kxr)[None, None, :]
        self.ky = (1j * kyr)[None, :, None]
        self.kz = (1j * kzr)[:, None, None]
        self.Lx = 2 * np.pi / p.alpha_x
        self.Ly = 2 * np.pi / p.alpha_y
        self.Lz = 2 * np.pi / p.alpha_z
        # variables.f90:273
        self.scalemodes = 1.0 / float(nx * ny * nz)
        # |k| as the spectral loops compute it (rhs.f90:70-72)
        self.absk = np.sqrt(np.real(np.conj(self.kx) * self.kx
                                    + np.conj(self.ky) * self.ky
                                    + np.conj(self.kz) * self.kz))
        self.absk = np.broadcast_to(self.absk, (nz, ny, self.nxh)).copy()
        # variables.f90:112-123
        if p.spherical:
            self.nspec = int(((nx / 2.0) * (2.0 * p.alpha_x / 3.0)) / p.Deltak) - 1
        else:
            self.nspec = int(np.sqrt(((nx / 2.0) * (2.0 * p.alpha_x / 3.0)) ** 2
                                     + ((ny / 2.0) * (2.0 * p.alpha_y / 3.0)) ** 2
                                     + ((nz / 2.0) * (2.0 * p.alpha_z / 3.0)) ** 2)
                             / p.Deltak) - 1
        # physical coordinates, variables.f90:235-266: x(ind) = i*Lx/Nx, i = -Nx/2..Nx/2-1
        self.x = np.array([i * self.Lx / nx for i in range(-nx // 2, nx // 2)])
        self.y = np.array([i * self.Ly / ny for i in range(-ny // 2, ny // 2)])
        self.z = np.array([i * self.Lz / nz for i in range(-nz // 2, nz // 2)])
        # kx == 0 plane flag (index 0 and the Nyquist index, Q1)
        self.kx_zero = np.broadcast_to((kxr == 0.0)[None, None, :], (nz, ny, self.nxh))
        self.all_zero = np.broadcast_to((kxr == 0.0)[None, None, :]
                                        & (kyr == 0.0)[None, :, None]
                                        & (kzr == 0.0)[:, None, None], (nz, ny, self.nxh))

    # ---------------------------------------------------------------- FFTs
    def r2c(self, f):
        """p3dfft_ftran_r2c: unnormalised forward R2C (state.f90:60-62)."""
        return sfft.rfftn(f, axes=(-3, -2, -1), workers=WORKERS)

    def c2r(self, F):
        """p3dfft_btran_c2r: unnormalised backward C2R (state.f90:68-70)."""
        p = self.p
        return sfft.irfftn(F, s=(p.nz, p.ny, p.nx), axes=(-3, -2, -1),
                           norm="forward", workers=WORKERS)

    # ---------------------------------------------------------------- masks
    def dealias_mask(self, spherical_factor, strict=False):
        """Modes zeroed by the 2/3 rule.

        rhs.f90:74-88 (``spherical_factor`` 0.5, ``.ge.``), state.f90:186-199
        (``spherical_factor`` 2/3, ``.ge.``), rhsAdj.f90:131-136 (``strict``:
        ``.gt.``, no spherical branch, no k = 0 term)."""
        p = self.p
        ax, ay, az = np.abs(self.kx), np.abs(self.ky), np.abs(self.kz)
        cx = (p.nx / 2.0) * (2.0 * p.alpha_x / 3.0)
        cy = (p.ny / 2.0) * (2.0 * p.alpha_y / 3.0)
        cz = (p.nz / 2.0) * (2.0 * p.alpha_z / 3.0)
        if strict:
            m = (ax > cx) | (ay > cy) | (az > cz)
            return np.broadcast_to(m, self.absk.shape).copy()
        m = (ax >= cx) | (ay >= cy) | (az >= cz)
        if p.spherical:
            m = m | (ax ** 2.0 + ay ** 2.0 + az ** 2.0
                     >= ((p.nx / 2.0) * spherical_factor * p.alpha_x) ** 2)
        m = np.broadcast_to(m, self.absk.shape) | self.all_zero
        return m.copy()


# ======================================================================= rhs.f90
def rhs_int_fact(g: Grid, dt: float):
    """rhs.f90:8-16: intFact = exp((nu*(kx*kx+ky*ky+kz*kz) + Q)*dt) (real-valued)."""
    p = g.p
    kk = g.kx * g.kx + g.ky * g.ky + g.kz * g.kz
    return np.real(np.exp((p.nu * kk + p.Q) * dt))


def rhs_eband(g: Grid, uh):
    """rhs.f90:137-168: band energy, kx = 0 plane half weighted, |k| <= kCutOff."""
    p = g.p
    scalex = np.where(g.kx_zero, 0.5, 1.0)
    inband = g.absk <= p.kCutOff
    e2 = (np.abs(uh[0]) ** 2 * scalex + np.abs(uh[1]) ** 2 * scalex
          + np.abs(uh[2]) ** 2 * scalex)
    return float(np.sum(e2[inband]) * g.scalemodes ** 2)


def state_derivatives(g: Grid, uh):
    """state.f90:456-500: grad[i][j] = d u_i / d x_j from 9 C2R of uhat*k_j*scalemodes."""
    s = g.scalemodes
    ks = (g.kx, g.ky, g.kz)
    return [[g.c2r(uh[i] * ks[j] * s) for j in range(3)] for i in range(3)]


def state_vorticity(d):
    """state.f90:502-515."""
    return (d[2][1] - d[1][2], d[0][2] - d[2][0], d[1][0] - d[0][1])


def rhs_nonlinear(g: Grid, uh, return_eband=False):
    """rhs.f90:18-135: rotational-form nonlinear term of uhattemp ``uh``.

    Returns N (3, nz, ny, nxh); 15 transforms as the reference."""
    p = g.p
    s = g.scalemodes
    eband = rhs_eband(g, uh) if p.bandlim else 0.0          # rhs.f90:22-24
    d = state_derivatives(g, uh)                            # rhs.f90:26
    ox, oy, oz = state_vorticity(d)                         # rhs.f90:27
    ut = g.c2r(uh[0].copy())                                # rhs.f90:30-37 (x N^3)
    vt = g.c2r(uh[1].copy())
    wt = g.c2r(uh[2].copy())
    nu_ = g.r2c((oy * wt - oz * vt) * s)                    # rhs.f90:39-47
    nv_ = g.r2c((oz * ut - ox * wt) * s)                    # rhs.f90:49-56
    nw_ = g.r2c((ox * vt - oy * ut) * s)                    # rhs.f90:58-65
    mask = g.dealias_mask(0.5)                              # rhs.f90:74-88
    kx, ky, kz = g.kx, g.ky, g.kz
    kk = kx * kx + ky * ky + kz * kz
    with np.errstate(divide="ignore", invalid="ignore"):
        phat = -1.0 * (kx * nu_ + ky * nv_ + kz * nw_) / kk  # rhs.f90:101-106
    phat = np.where(g.all_zero, 0.0, phat)                  # rhs.f90:95-98
    band = (g.absk <= p.kCutOff) if p.bandlim else np.zeros(g.absk.shape, bool)
    fc = (p.Pin / (2.0 * eband)) if p.bandlim else 0.0
    out = np.empty((3,) + g.absk.shape, np.complex128)
    for c, (n_, kc) in enumerate(((nu_, kx), (nv_, ky), (nw_, kz))):
        base = -n_ - kc * phat                              # rhs.f90:120-128
        forced = base + fc * uh[c] if p.bandlim else base   # rhs.f90:110-118
        out[c] = np.where(band, forced, base)
    out[:, mask] = 0.0                                      # rhs.f90:90-92
    if return_eband:
        return out, eband
    return out


# ================================================================ steppers
def heun_step(g: Grid, uh, dt, force=None):
    """dnsboxheun.f90:85-126: IF predictor-corrector (Heun).  ``force`` is an
    optional fixed spectral forcing added to N (the Kolmogorov forcing of the
    adjoint configuration; not in the reference)."""
    IF = rhs_int_fact(g, dt)
    n1 = rhs_nonlinear(g, uh)                               # :85
    if force is not None:
        n1 = n1 + force
    ut = IF * (uh + dt * n1)                                # :91-92
    un = IF * (uh + dt * n1 * 0.5)                          # :95-96
    n2 = rhs_nonlinear(g, ut)                               # :117
    if force is not None:
        n2 = n2 + force
    return un + dt * n2 * 0.5                               # :122-124


def semi_implicit_step(g: Grid, uh, dt, c=0.5, tol=1e-10, max_iter=50):
    """dnsboximplicit.f90:88-181: the semi-implicit step with fixed-point
    iterations (implicitness ``c``, parameters.f90:47; tolerance ``tol``,
    parameters.f90:26).  The driver's ``rhsFix`` and ``rhstStepFact`` are
    defined nowhere in the reference; they are restated here as the theta
    scheme of the Crank-Nicolson solver nsbox.f90:192-221 with ``c`` the
    implicitness of both the linear and the nonlinear term:
      fac = 1 / (1/dt - c L),  fix = (1/dt + (1 - c) L) u_n,  L = nu k.k + Q
      u^0 = fac (fix + N(u_n))                                       (:112-120)
      u^(k+1) = fac (fix + c N(u^k) + (1 - c) N(u_n))               (:149-162)
    until sum_i max |u_i^(k+1) - u_i^k| <= tol on the (unnormalised) spectral
    values (:164-173), at most ``max_iter`` iterations; then state_project
    (:177).  Returns (new state, iterations)."""
    p = g.p
    L = p.nu * np.real(g.kx * g.kx + g.ky * g.ky + g.kz * g.kz) + p.Q
    fac = 1.0 / (1.0 / dt - c * L)
    fix = (1.0 / dt + (1.0 - c) * L) * uh
    n0 = rhs_nonlinear(g, uh)                               # :93
    u = fac * (fix + n0)                                    # :112-120
    it = 0
    while it < max_iter:
        it += 1
        nk = rhs_nonlinear(g, u)                            # :137
        un = fac * (fix + c * nk + (1.0 - c) * n0)          # :149-162
        chg = sum(float(np.max(np.abs(un[i] - u[i]))) for i in range(3))   # :164-173
        u = un
        if chg <= tol:
            break
    return state_project(g, u), it                          # :177


class AB2Stepper:
    """dnsbox.f90:87-218 (timestepper = 2): PC first step, then IF-AB2.

    ``ab2="reference"`` keeps the literal coefficients of dnsbox.f90:93-104
    (c2 = 0.5*(t_n - dt - t_{n-1}), Q2); ``ab2="standard"`` uses the
    variable-step IF-AB2 c1 = dt*(1 + dt/(2 h)), c2 = -dt^2/(2 h),
    h = t_n - t_{n-1}."""

    def __init__(self, g: Grid):
        self.g = g
        self.n = 0
        self.times = [0.0]
        self.nold = None

    def step(self, uh, dt):
        g, p = self.g, self.g.p
        self.n += 1
        kk = g.kx * g.kx + g.ky * g.ky + g.kz * g.kz
        if self.n == 1:
            IF = rhs_int_fact(g, dt)
            n1 = rhs_nonlinear(g, uh)                        # :89
            ut = IF * (uh + dt * n1)                         # :95-96
            un = IF * (uh + dt * n1 * 0.5)                   # :99-101
            self.nold = n1                                   # :121-125
            n2 = rhs_nonlinear(g, ut)                        # :130
            un = un + dt * n2 * 0.5                          # :135-137
        else:
            tn, tm = self.times[-1], self.times[-2]
            n1 = rhs_nonlinear(g, uh)                        # :146
            IF = rhs_int_fact(g, dt)
            if p.ab2 == "reference":
                c1 = 0.5 * (tn + tn + dt - 2.0 * tm)         # :151
                c2 = 0.5 * (2.0 * tn - tn - dt - tm)         # :156
            else:
                h = tn - tm
                c1 = dt * (1.0 + dt / (2.0 * h))
                c2 = -dt * dt / (2.0 * h)
            e1 = np.real(np.exp((p.nu * kk + p.Q) * dt))
            e2 = np.real(np.exp((p.nu * kk + p.Q) * (dt + tn - tm)))
            un = IF * uh + c1 * e1 * n1 + c2 * e2 * self.nold  # :150-161
            self.nold = n1                                   # :210-212
        self.times.append(self.times[-1] + dt)               # :218
        return un


# ======================================================== state.f90 operators
def state_project(g: Grid, uh):
    """state.f90:120-179 (eps = 0: never assigned in the rhs.f90 build)."""
    kx, ky, kz = g.kx, g.ky, g.kz
    u, v, w = uh
    with np.errstate(divide="ignore", invalid="ignore"):
        kk = kx * kx + ky * ky + kz * kz
        nu_ = u - kx * kx * u / kk - kx * ky * v / kk - kx * kz * w / kk
        nv_ = v - ky * kx * u / kk - ky * ky * v / kk - ky * kz * w / kk
        nw_ = w - kz * kx * u / kk - kz * ky * v / kk - kz * kz * w / kk
    out = np.stack([nu_, nv_, nw_])
    keep = np.broadcast_to(g.all_zero, out.shape[1:])
    out[:, keep] = uh[:, keep]                              # :127-130 (cycle)
    return out


def state_dealias(g: Grid, uh):
    """state.f90:181-209."""
    out = uh.copy()
    out[:, g.dealias_mask(2.0 / 3.0)] = 0.0
    return out


def _shell_index(g: Grid):
    """state.f90:363-367: nearest-window index nk of |k|."""
    p = g.p
    absk = g.absk
    base = np.floor(absk / p.Deltak)        # int() of a non-negative number
    return np.where(absk < base + 0.5 * p.Deltak, base, base + 1).astype(np.int64)


def state_spectrum(g: Grid, uh, mode=None):
    """state.f90:350-411 (``mode="mpi"``) or single/state.f90:191-230 (``"single"``).

    Returns (Espec[1..Nspec] as an array of length Nspec, EZero, EOne, Esqrt2)."""
    p = g.p
    mode = mode or p.spectrum_mode
    e2 = np.abs(uh[0]) ** 2 + np.abs(uh[1]) ** 2 + np.abs(uh[2]) ** 2
    absk = g.absk
    nk = _shell_index(g)
    espec = np.zeros(g.nspec)
    if mode == "mpi":
        ezero = float(np.sum(e2[absk == 0]))                         # :369-374
        eone = float(np.sum(e2[absk == 1.0]))                        # :376-381
        esq2 = float(np.sum(e2[absk - np.sqrt(2.0) < 1.0e-9]))       # :383-388
        sel = (nk < g.nspec) & (nk != 0)                             # :390
        np.add.at(espec, nk[sel] - 1, e2[sel] * g.scalemodes ** 2 / p.Deltak)
    else:
        w = np.where(g.kx_zero, 0.5, 1.0)
        ezero = float(np.sum((e2 * w)[absk == 0]))
        eone = 0.0
        esq2 = 0.0
        sel = (nk <= g.nspec) & (nk != 0)
        np.add.at(espec, nk[sel] - 1,
                  (e2 * w)[sel] * g.scalemodes ** 2 / p.Deltak)
    return espec, ezero, eone, esq2


def state_kinetic(g: Grid, uh):
    """state.f90:429-454: E = scalemodes^2 * sum(w |uhat|^2), w = 1/2 on kx = 0."""
    w = np.where(g.kx_zero, 0.5, 1.0)
    e = (np.abs(uh[0]) ** 2 * w + np.abs(uh[1]) ** 2 * w + np.abs(uh[2]) ** 2 * w)
    return float(np.sum(e) * g.scalemodes ** 2)


def state_dissipation(g: Grid, uh):
    """state.f90:517-544: nu * scalemodes * sum over the grid of |grad u|^2 (9 C2R)."""
    d = state_derivatives(g, uh)
    tot = 0.0
    for i in range(3):
        for j in range(3):
            tot += float(np.sum(d[i][j] * d[i][j]))
    return tot * g.p.nu * g.scalemodes


def dissipation_spectral(g: Grid, uh):
    """Parseval form of state_dissipation: nu * s^2 * sum_full |k|^2 |uhat|^2.

    The half-spectrum weight is 1 on the kx = 0 and Nyquist planes, 2 elsewhere."""
    wfull = np.where(g.kx_zero, 1.0, 2.0)
    e2 = np.abs(uh[0]) ** 2 + np.abs(uh[1]) ** 2 + np.abs(uh[2]) ** 2
    return float(g.p.nu * g.scalemodes ** 2 * np.sum(wfull * g.absk ** 2 * e2))


def state_divergence(g: Grid, uh):
    """state.f90:413-427: signed max of u_x + v_y + w_z on the grid."""
    s = g.scalemodes
    div = (g.c2r(uh[0] * g.kx * s) + g.c2r(uh[1] * g.ky * s) + g.c2r(uh[2] * g.kz * s))
    return float(np.max(div))


def state_uhat2u(g: Grid, uh):
    """state.f90:82-96: physical velocity, C2R times scalemodes."""
    return np.stack([g.c2r(uh[c].copy()) * g.scalemodes for c in range(3)])


def state_u2uhat(g: Grid, u):
    """state.f90:74-80."""
    return np.stack([g.r2c(u[c]) for c in range(3)])


def io_courant(g: Grid, u, dt):
    """io.f90:664-676 on a physical velocity ``u`` (3, nz, ny, nx)."""
    p = g.p
    return (np.max(np.abs(u[0])) * dt / (g.Lx / p.nx)
            + np.max(np.abs(u[1])) * dt / (g.Ly / p.ny)
            + np.max(np.abs(u[2])) * dt / (g.Lz / p.nz))


def set_time_step(g: Grid, dt, courant):
    """dnsboxheun.f90:227-246: dt <- ((Cmin + Cmax)/(2 C)) dt, capped at tStepMax.

    Returns the new dt and the new Courant number (io_Courant re-evaluated,
    which is linear in dt)."""
    p = g.p
    new = ((p.courant_max + p.courant_min) / (2.0 * courant)) * dt
    if new > p.dt_max:
        new = p.dt_max
    return new, courant * new / dt


def needs_time_step(g: Grid, dt, courant):
    """dnsboxheun.f90:153-155."""
    p = g.p
    return (not p.tstep_fix) and (courant > p.courant_max
                                  or (courant < p.courant_min and dt < p.dt_max))


YOFFE_C = (8.0e-2, 2.0, 8.2352309e-2, 2.0)   # state.f90:218-221 (C1..C4)


def state_init_rand(g: Grid, noise):
    """state.f90:211-285 (Yoffe 2012, s. 2.2.5) from a given physical noise
    field ``noise`` (3, nz, ny, nx): R2C, dealias, project, spectrum, and every
    mode multiplied by sqrt(C1 (nk dk)^C2 exp(-C3 (nk dk)^C4) / Espec(nk)) with
    nk the nearest shell; nk = 0 and nk >= Nspec are zeroed (:251-283).
    Returns the spectral state (the reference continues with state_uhat2u)."""
    p = g.p
    uh = state_project(g, state_dealias(g, state_u2uhat(g, noise)))   # :240-243
    espec, *_ = state_spectrum(g, uh)                                  # :244
    nk = _shell_index(g)                                               # :249-254
    c1, c2, c3, c4 = YOFFE_C
    ok = (nk != 0) & (nk < g.nspec)                                    # :256
    kn = np.where(ok, nk, 1) * p.Deltak
    fac = np.where(ok, np.sqrt(c1 * kn ** c2 * np.exp(-c3 * kn ** c4)
                               / np.where(ok, espec[np.where(ok, nk, 1) - 1], 1.0)), 0.0)
    return uh * fac


def beltrami(g: Grid, t):
    """state.f90:287-307 (u, v, w at time t), physical layout [z, y, x]."""
    nu = g.p.nu
    f = np.sqrt(3.0)
    Z, Y, X = np.meshgrid(g.z, g.y, g.x, indexing="ij")
    dec = np.exp(-(f ** 2) * t * nu)
    u = -0.5 * (f * np.cos(X) * np.sin(Y) * np.sin(Z) + np.sin(X) * np.cos(Y) * np.cos(Z)) * dec
    v = 0.5 * (f * np.sin(X) * np.cos(Y) * np.sin(Z) - np.cos(X) * np.sin(Y) * np.cos(Z)) * dec
    w = 1.0 * np.cos(X) * np.cos(Y) * np.sin(Z) * dec
    return np.stack([u, v, w])


# ============================================================== rhsAdj.f90
def adj_rhs_nonlinear(g: Grid, uh):
    """rhsAdj.f90:64-175: convective-form N, ``.gt.`` dealias, eps = 1e-13 at k = 0."""
    s = g.scalemodes
    d = state_derivatives(g, uh)                                     # :68
    ut, vt, wt = (g.c2r(uh[c].copy()) for c in range(3))             # :75-77 (Q8)
    n = [g.r2c((ut * d[c][0] + vt * d[c][1] + wt * d[c][2]) * s) for c in range(3)]
    return _adj_finish(g, n, n)


def _adj_finish(g: Grid, n, n_for_phat, phat_mode="intent"):
    """Spectral loop of rhsAdj.f90:128-169 / 311-352."""
    kx, ky, kz = g.kx, g.ky, g.kz
    mask = g.dealias_mask(0.0, strict=True)
    eps = np.where(g.all_zero, 0.1 ** 13, 0.0)
    kk = kx * kx + ky * ky + kz * kz + eps
    phat = -1.0 * (kx * n_for_phat[0] + ky * n_for_phat[1] + kz * n_for_phat[2]) / kk
    use = phat if phat_mode == "intent" else 0.0
    out = np.stack([-n[0] - kx * use, -n[1] - ky * use, -n[2] - kz * use])
    out[:, mask] = 0.0
    return out


def adj_rhsupptilde(g: Grid, uh):
    """rhsAdj.f90:177-213: r~ = H^{-1} ((nu k.k + Q) uhat + N(uhat))."""
    p = g.p
    N = adj_rhs_nonlinear(g, uh)
    kk = g.kx * g.kx + g.ky * g.ky + g.kz * g.kz
    factor = 1.0 / (1.0 - np.real(kk)) if p.hminone else 1.0
    return factor * ((p.nu * kk + p.Q) * uh + N)


def adj_nonlinear_part(g: Grid, uh, rt, phat_mode=None):
    """rhsAdj.f90:261-354 given r~ = ``rt``: -P_d[F((grad r~)^T u + (u.grad) r~)]."""
    s = g.scalemodes
    phat_mode = phat_mode or g.p.adj_phat
    dr = state_derivatives(g, rt)                                    # :215-259
    ut, vt, wt = (g.c2r(uh[c].copy()) for c in range(3))             # :267-269
    uu = (ut, vt, wt)
    n = []
    for c in range(3):
        acc = (dr[0][c] * ut + dr[1][c] * vt + dr[2][c] * wt          # (grad r~)^T u
               + dr[c][0] * ut + dr[c][1] * vt + dr[c][2] * wt)       # (u.grad) r~
        n.append(g.r2c(acc * s))                                     # :271-309
    del uu
    return _adj_finish(g, n, n, phat_mode)


def rhs_adj(g: Grid, uh):
    """rhsAdj.f90:356-381: returns (r~, rhsadj)."""
    p = g.p
    rt = adj_rhsupptilde(g, uh)
    nadj = adj_nonlinear_part(g, uh, rt)
    kk = g.kx * g.kx + g.ky * g.ky + g.kz * g.kz
    return rt, (p.nu * kk + p.Q) * rt + nadj


# ===================================================== exact adjoint (VJP)
def half_weight(g: Grid):
    """Half-spectrum multiplicity W: 1 on the kx = 0 and Nyquist planes, 2 elsewhere."""
    return np.where(g.kx_zero, 1.0, 2.0)


def rhs_nonlinear_vjp(g: Grid, uh, gout):
    """Exact transpose of the linearised rhs_nonlinear (bandlim off), with respect
    to the Euclidean inner product on the (Re, Im) parts of the half spectrum.

    N(uh) = -D P R2C(omega x u) with u = C2R(uh) s, omega = C2R(ik x uh) s.
    Transposes: C2R^T = W * R2C, R2C^T = C2R(. / W), the curl is Hermitian."""
    s = g.scalemodes
    W = half_weight(g)
    k = (g.kx, g.ky, g.kz)
    mask = g.dealias_mask(0.5)
    # h = -P(D g)
    gm = np.where(mask[None], 0.0, gout)
    kk = k[0] * k[0] + k[1] * k[1] + k[2] * k[2]
    with np.errstate(divide="ignore", invalid="ignore"):
        kdotg = (k[0] * gm[0] + k[1] * gm[1] + k[2] * gm[2]) / kk
    kdotg = np.where(g.all_zero, 0.0, kdotg)
    h = np.stack([-(gm[c] - k[c] * kdotg) for c in range(3)])
    phi = np.stack([g.c2r(h[c] / W) for c in range(3)])
    u = np.stack([g.c2r(uh[c].copy()) * s for c in range(3)])
    curl = (k[1] * uh[2] - k[2] * uh[1], k[2] * uh[0] - k[0] * uh[2],
            k[0] * uh[1] - k[1] * uh[0])
    om = np.stack([g.c2r(curl[c]) * s for c in range(3)])
    uxphi = np.cross(u, phi, axis=0)
    phixom = np.cross(phi, om, axis=0)
    psi = np.stack([s * W * g.r2c(uxphi[c]) for c in range(3)])
    grad_u = np.stack([s * W * g.r2c(phixom[c]) for c in range(3)])
    # curl transpose: (ik x)^T = (ik x) (Hermitian)
    curl_t = np.stack([k[1] * psi[2] - k[2] * psi[1], k[2] * psi[0] - k[0] * psi[2],
                       k[0] * psi[1] - k[1] * psi[0]])
    return curl_t + grad_u


def heun_step_vjp(g: Grid, uh, dt, gout, force=None):
    """Transpose of the linearised IF-Heun step (heun_step at fixed dt, bandlim
    off) at uh applied to gout, Euclidean on (Re, Im) of the half spectrum.
    With S(u) = IF u + dt/2 IF N(u) + dt/2 N(u*), u* = IF (u + dt N(u)) and IF
    real and diagonal:
        a = N'(u*)^T (dt/2 gout),
        S'(u)^T gout = IF (gout + a) + N'(u)^T (IF (dt/2 gout + dt a))."""
    IF = rhs_int_fact(g, dt)
    n1 = rhs_nonlinear(g, uh)
    if force is not None:
        n1 = n1 + force
    ut = IF * (uh + dt * n1)
    a = rhs_nonlinear_vjp(g, ut, 0.5 * dt * gout)
    return IF * (gout + a) + rhs_nonlinear_vjp(g, uh, IF * (0.5 * dt * gout + dt * a))


def orbit_residual_grad(g: Grid, u0, dt, nsteps, force=None):
    """Periodic-orbit residual J(u0) = 1/2 <(u(T) - u0)^2> (mean square over
    the physical grid, = 1/2 s^2 sum_half W |r|^2 with r = u(T) - u0 and T =
    nsteps dt of fixed-dt IF-Heun) and its gradient (Euclidean on Re/Im of the
    half spectrum): grad = (Phi'^T - I) (s^2 W r), Phi' backpropagated through
    the stored states."""
    s2 = g.scalemodes ** 2
    W = half_weight(g)
    states = [u0]
    for _ in range(nsteps):
        states.append(heun_step(g, states[-1], dt, force))
    r = states[-1] - u0
    J = 0.5 * s2 * float(np.sum(W * np.abs(r) ** 2))
    gc = s2 * W * r
    gb = gc
    for n in range(nsteps - 1, -1, -1):
        gb = heun_step_vjp(g, states[n], dt, gb, force)
    return J, gb - gc


# ================================================================ drivers
def drive(g: Grid, uh, nsteps, dt, stepper="heun", cfl=False):
    """Time loop of dnsboxheun.f90:81-191 / dnsbox.f90:81-218 without I/O.

    With ``cfl`` the Courant number is taken from the current velocity every
    step (quirk Q5: the reference uses a copy refreshed every iSaveRate1
    steps) and set_time_step is applied before the first step (as
    dnsboxheun.f90:69-73) and whenever it leaves [Cmin, Cmax]."""
    recs = []
    ab2 = AB2Stepper(g) if stepper == "ab2" else None
    first = True
    for _ in range(nsteps):
        umax = np.abs(state_uhat2u(g, uh)).reshape(3, -1).max(axis=1)
        C = io_courant(g, state_uhat2u(g, uh), dt)
        if cfl and (first or needs_time_step(g, dt, C)):
            dt, C = set_time_step(g, dt, C)
        first = False
        uh = heun_step(g, uh, dt) if ab2 is None else ab2.step(uh, dt)
        recs.append(dict(dt=dt, courant=C, umax=umax, ekin=state_kinetic(g, uh),
                         dissipation=dissipation_spectral(g, uh)))
    return uh, recs
