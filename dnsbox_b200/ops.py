"""PyTorch-facing operators of the dnsbox time step (one GPU).

``Box`` owns one ``dnsbox_ctx`` of libdnsbox_gpu.so and mirrors the reference
operator surface (names of rhs.f90 / state.f90 / io.f90 / the drivers), taking
and returning CUDA tensors:

  =====================  ==============================================
  Box method             reference routine
  =====================  ==============================================
  rhs_nonlinear          rhs_nonlinear + rhs_Eband (rhs.f90:18-168)
  set_dt / get_dt        rhs_int_fact (rhs.f90:8-16), dt of variables.f90
  step                   IF Heun loop (dnsboxheun.f90:81-191) or IF-AB2
                         (dnsbox.f90:87-218) with CFL control
  project / dealias      state_project / state_dealias (state.f90:120-209)
  spectrum               state_spectrum (state.f90:350-411)
  kinetic / dissipation  state_kinetic / state_dissipation (state.f90:429-544)
  courant                io_Courant (io.f90:664-676)
  divergence             state_divergence (state.f90:413-427)
  r2c / c2r              p3dfft_ftran_r2c / p3dfft_btran_c2r
  =====================  ==============================================

Spectral tensors are (3, nz, ny, nx//2+1) complex128 (FP64) or complex64
(FP32), contiguous, on the Box's device.  Every call is issued on the current
torch CUDA stream.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .grid import nspec as _nspec

PRECISION = {"fp64": 0, "fp32": 1, "tc_split": 2}
STEPPER = {"heun": 0, "ab2": 1, "semi_implicit": 2}
TC_KERNELS = ("tma", "cp.async", "simt")   # per strided pass of the tensor-core form
X_KERNELS = ("default", "block", "warp", "warp-registers", "warp-registers-128")   # the fused x pass
AB2_MODE = {"reference": 0, "standard": 1}
SPECTRUM_MODE = {"mpi": 0, "single": 1}
ADJ_PHAT = {"intent": 0, "literal": 1}


def _ptr(t: torch.Tensor):
    return ctypes.c_void_p(t.data_ptr())


class Box:
    """One periodic box on one GPU (replaces ``var_init``, variables.f90:99-280)."""

    def __init__(self, n=None, *, nx=None, ny=None, nz=None, precision="fp64", stepper="heun",
                 ab2="reference", nu=0.005, Q=0.0, kCutOff=2.0, Pin=0.1, Deltak=1.0,
                 courant_min=0.15, courant_max=0.2, dt_max=1.0e-2, dt=1.0e-3, bandlim=True,
                 spherical=False, tstep_fix=False, hminone=True, spectrum_mode="mpi",
                 adj_phat="intent", alpha=(1.0, 1.0, 1.0), device=None, nbatch=1, prune=True,
                 implicit_c=0.5, implicit_tol=1e-10, implicit_max_iter=50):
        if not torch.cuda.is_available():
            raise RuntimeError("dnsbox_b200 needs a CUDA device (there is no CPU path)")
        lib = _lib.load()
        nx = nx or n
        ny = ny or n
        nz = nz or n
        if device is None:
            device = torch.cuda.current_device()
        self.device = torch.device("cuda", device)
        p = _lib.Params()
        lib.dnsbox_default_params(ctypes.byref(p))
        p.nx, p.ny, p.nz = nx, ny, nz
        p.precision = PRECISION[precision]
        p.stepper = STEPPER[stepper]
        p.ab2_mode = AB2_MODE[ab2]
        p.bandlim, p.spherical, p.tstep_fix, p.hminone = int(bandlim), int(spherical), int(tstep_fix), int(hminone)
        p.spectrum_mode = SPECTRUM_MODE[spectrum_mode]
        p.adj_phat = ADJ_PHAT[adj_phat]
        p.device = device
        p.nbatch = int(nbatch)
        p.no_prune = 0 if prune else 1
        p.alpha_x, p.alpha_y, p.alpha_z = alpha
        p.nu, p.Q, p.kCutOff, p.Pin, p.Deltak = nu, Q, kCutOff, Pin, Deltak
        p.courant_min, p.courant_max, p.dt_max, p.dt = courant_min, courant_max, dt_max, dt
        p.implicit_c, p.implicit_tol, p.implicit_max_iter = implicit_c, implicit_tol, int(implicit_max_iter)
        self.params = p
        self.nx, self.ny, self.nz = nx, ny, nz
        self.nxh = nx // 2 + 1
        self.nbatch = max(1, int(nbatch))
        self.precision = precision
        self.cdtype = torch.complex128 if precision == "fp64" else torch.complex64
        self.rdtype = torch.float64 if precision == "fp64" else torch.float32
        self.nspec = _nspec(nx, ny, nz, alpha, Deltak, spherical)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(lib.dnsbox_create(ctypes.byref(p), ctypes.byref(h)))
        self._h = h
        self._lib = lib

    # ---------------------------------------------------------------- plumbing
    @property
    def handle(self) -> int:
        """The dnsbox_ctx pointer, the context argument of torch.ops.dnsbox.*."""
        return int(self._h.value or 0)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.dnsbox_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _sync_stream(self):
        s = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self._lib.dnsbox_set_stream(self._h, ctypes.c_void_p(s)))

    def _check_state(self, t: torch.Tensor, name="uhat"):
        shape = self.spectral_shape()
        if t.shape != shape or t.dtype != self.cdtype or not t.is_contiguous() or t.device != self.device:
            raise ValueError(f"{name} must be a contiguous {self.cdtype} tensor of shape {shape} on "
                             f"{self.device}, got {tuple(t.shape)} {t.dtype} {t.device}")

    def spectral_shape(self):
        """(3, nz, ny, nxh), or (3, nbatch, nz, ny, nxh) for a batched Box."""
        if self.nbatch > 1:
            return (3, self.nbatch, self.nz, self.ny, self.nxh)
        return (3, self.nz, self.ny, self.nxh)

    def zeros(self):
        return torch.zeros(self.spectral_shape(), dtype=self.cdtype, device=self.device)

    def from_numpy(self, uh: np.ndarray) -> torch.Tensor:
        return torch.from_numpy(np.ascontiguousarray(uh)).to(self.device, self.cdtype)

    # ---------------------------------------------------------------- time step
    def set_dt(self, dt: float):
        _lib.check(self._lib.dnsbox_set_dt(self._h, float(dt)))

    def get_dt(self) -> float:
        v = ctypes.c_double()
        self._sync_stream()
        _lib.check(self._lib.dnsbox_get_dt(self._h, ctypes.byref(v)))
        return v.value

    def set_time(self, t: float):
        _lib.check(self._lib.dnsbox_set_time(self._h, float(t)))

    def get_time(self) -> float:
        v = ctypes.c_double()
        self._sync_stream()
        _lib.check(self._lib.dnsbox_get_time(self._h, ctypes.byref(v)))
        return v.value

    def reset_history(self):
        _lib.check(self._lib.dnsbox_reset_history(self._h))

    # ---------------------------------------------------------------- operators
    def rhs_nonlinear(self, uh: torch.Tensor, out: torch.Tensor | None = None, want_eband=True):
        self._check_state(uh)
        if out is None:
            out = torch.empty_like(uh)
        self._check_state(out, "out")
        self._sync_stream()
        eb = ctypes.c_double()
        _lib.check(self._lib.dnsbox_rhs_nonlinear(self._h, _ptr(uh), _ptr(out),
                                                  ctypes.byref(eb) if want_eband else None))
        return out, (eb.value if want_eband else None)

    def step(self, uh: torch.Tensor, nsteps: int = 1, diag: bool = True):
        """Advance ``uh`` in place by ``nsteps``; returns a list of per-step dicts."""
        self._check_state(uh)
        self._sync_stream()
        if not diag:
            _lib.check(self._lib.dnsbox_step(self._h, _ptr(uh), int(nsteps), None))
            return None
        recs = (_lib.Diag * (nsteps * self.nbatch))()
        _lib.check(self._lib.dnsbox_step(self._h, _ptr(uh), int(nsteps), recs))
        return self._records(recs, nsteps)

    def _records(self, recs, nsteps):
        out = [dict(t=r.t, dt=r.dt, ekin=r.ekin, dissipation=r.dissipation,
                    production_literal=r.production_literal, injected_power=r.injected_power,
                    courant=r.courant, umax=tuple(r.umax), eband=r.eband, step=r.step) for r in recs]
        if self.nbatch == 1:
            return out
        return [out[i * self.nbatch:(i + 1) * self.nbatch] for i in range(nsteps)]

    def diag_read(self, nrecent: int):
        """Step records of the last nrecent steps (kept on the device)."""
        self._sync_stream()
        recs = (_lib.Diag * (nrecent * self.nbatch))()
        _lib.check(self._lib.dnsbox_diag_read(self._h, int(nrecent), recs))
        return self._records(recs, nrecent)

    def set_batch_nu(self, nus):
        v = np.ascontiguousarray(np.broadcast_to(np.asarray(nus, np.float64), (self.nbatch,)))
        _lib.check(self._lib.dnsbox_set_batch_nu(self._h, v.ctypes.data_as(_lib._DP)))

    def project(self, uh):
        self._check_state(uh)
        self._sync_stream()
        _lib.check(self._lib.dnsbox_project(self._h, _ptr(uh)))
        return uh

    def dealias(self, uh):
        self._check_state(uh)
        self._sync_stream()
        _lib.check(self._lib.dnsbox_dealias(self._h, _ptr(uh)))
        return uh

    def spectrum(self, uh):
        self._check_state(uh)
        self._sync_stream()
        es = np.zeros(self.nspec)
        e0, e1, e2 = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _lib.check(self._lib.dnsbox_spectrum(self._h, _ptr(uh), es.ctypes.data_as(_lib._DP),
                                             ctypes.byref(e0), ctypes.byref(e1), ctypes.byref(e2)))
        return es, e0.value, e1.value, e2.value

    def _scalar(self, fn, uh):
        self._check_state(uh)
        self._sync_stream()
        v = ctypes.c_double()
        _lib.check(fn(self._h, _ptr(uh), ctypes.byref(v)))
        return v.value

    def kinetic(self, uh):
        return self._scalar(self._lib.dnsbox_kinetic, uh)

    def dissipation(self, uh):
        return self._scalar(self._lib.dnsbox_dissipation, uh)

    def divergence(self, uh):
        return self._scalar(self._lib.dnsbox_divergence, uh)

    def eband(self, uh):
        return self._scalar(self._lib.dnsbox_eband, uh)

    def courant(self, uh, dt):
        self._check_state(uh)
        self._sync_stream()
        c = ctypes.c_double()
        m = (ctypes.c_double * 3)()
        _lib.check(self._lib.dnsbox_courant(self._h, _ptr(uh), float(dt), ctypes.byref(c), m))
        return c.value, tuple(m)

    # ---------------------------------------------------------------- adjoint
    def set_forcing(self, f: torch.Tensor | None):
        """Fixed spectral forcing added to the nonlinear term (None clears).
        The Box keeps a reference so the memory stays valid."""
        if f is not None:
            self._check_state(f, "forcing")
        self._force = f
        _lib.check(self._lib.dnsbox_set_forcing(self._h, _ptr(f) if f is not None else None))

    def rhs_adj(self, uh):
        """rhsAdj (rhsAdj.f90:356-381): returns (r~, rhsadj)."""
        self._check_state(uh)
        rt, out = torch.empty_like(uh), torch.empty_like(uh)
        self._sync_stream()
        _lib.check(self._lib.dnsbox_rhs_adj(self._h, _ptr(uh), _ptr(rt), _ptr(out)))
        return rt, out

    def rhs_nonlinear_vjp(self, uh, g):
        """Exact transpose of the linearised rhs_nonlinear at uh applied to g."""
        self._check_state(uh)
        g = g.contiguous()
        self._check_state(g, "g")
        out = torch.empty_like(uh)
        self._sync_stream()
        _lib.check(self._lib.dnsbox_rhs_nonlinear_vjp(self._h, _ptr(uh), _ptr(g), _ptr(out)))
        return out

    def residual(self, uh) -> float:
        self._check_state(uh)
        self._sync_stream()
        v = ctypes.c_double()
        _lib.check(self._lib.dnsbox_residual(self._h, _ptr(uh), ctypes.byref(v)))
        return v.value

    def residual_grad(self, uh):
        self._check_state(uh)
        grad = torch.empty_like(uh)
        self._sync_stream()
        v = ctypes.c_double()
        _lib.check(self._lib.dnsbox_residual_grad(self._h, _ptr(uh), _ptr(grad), ctypes.byref(v)))
        return v.value, grad

    def adjoint_descent(self, uh, niter, alpha=1.0):
        """niter descent iterations on J in place; returns (J history, step length)."""
        self._check_state(uh)
        self._sync_stream()
        hist = np.full(niter + 1, np.nan)
        a = ctypes.c_double(alpha)
        _lib.check(self._lib.dnsbox_adjoint_descent(self._h, _ptr(uh), int(niter),
                                                    hist.ctypes.data_as(_lib._DP), ctypes.byref(a)))
        return hist, a.value

    def sync(self):
        """Waits for the work queued on this Box and raises if a device-side
        wait gave up (a tensor-core pass whose output is then invalid)."""
        _lib.check(self._lib.dnsbox_sync(self._h))

    def init_yoffe(self, noise: torch.Tensor | None = None, seed: int = 0) -> torch.Tensor:
        """state_init_rand (state.f90:211-285) on the device: from the physical
        noise field (3, nz, ny, nx) in the Box's real dtype, or drawn from seed."""
        if noise is not None:
            noise = noise.contiguous()
            assert noise.shape == (3, self.nz, self.ny, self.nx) and noise.dtype == self.rdtype
        uh = self.zeros()
        self._sync_stream()
        _lib.check(self._lib.dnsbox_init_yoffe(self._h, _ptr(noise) if noise is not None else None,
                                               ctypes.c_uint64(seed), _ptr(uh)))
        return uh

    def init_beltrami(self, t: float = 0.0) -> torch.Tensor:
        """state_init_analytic (state.f90:287-307) at time t, as a spectral state."""
        uh = self.zeros()
        self._sync_stream()
        _lib.check(self._lib.dnsbox_init_beltrami(self._h, float(t), _ptr(uh)))
        return uh

    def set_step_projection(self, on: bool = True):
        """Project and dealias the state after every step (dnsboxband.f90:142-143)."""
        _lib.check(self._lib.dnsbox_set_step_projection(self._h, int(bool(on))))

    # ---------------------------------------------------------- kernel schedule
    @staticmethod
    def _sched_dict(sc, tc=True):
        return {"tc_kernel": [TC_KERNELS[v] if tc else "simt" for v in sc.tc_kernel[:3]],
                "z_fwd_kernel": "tma" if sc.tc_kernel[3] else "simt",
                "x_kernel": X_KERNELS[sc.x_kernel], "tuned": bool(sc.tuned),
                "ms_default": sc.ms_default, "ms_tuned": sc.ms_tuned}

    def schedule(self) -> dict:
        sc = _lib.Schedule()
        _lib.check(self._lib.dnsbox_get_schedule(self._h, ctypes.byref(sc)))
        return self._sched_dict(sc, self.precision == "tc_split")

    def set_schedule(self, tc_kernel=(0, 0, 0), x_kernel=0, z_fwd_tma=False):
        """tc_kernel: per pass A, B, D of the tensor-core form, 0 / "tma", 1 /
        "cp.async" or 2 / "simt"; x_kernel 0 .. 4 (or its name); z_fwd_tma: pass E1 on the
        TMA tensor-core kernel."""
        sc = _lib.Schedule()
        for i in range(3):
            v = tc_kernel[i]
            sc.tc_kernel[i] = TC_KERNELS.index(v) if isinstance(v, str) else int(v)
        sc.tc_kernel[3] = int(bool(z_fwd_tma))
        sc.x_kernel = X_KERNELS.index(x_kernel) if isinstance(x_kernel, str) else int(x_kernel)
        _lib.check(self._lib.dnsbox_set_schedule(self._h, ctypes.byref(sc)))

    def autotune(self, uh: torch.Tensor, nsteps: int = 4) -> dict:
        """Times the candidate kernels of every pass on a copy of uh and keeps
        the fastest (cached for this device and shape)."""
        self._check_state(uh)
        self._sync_stream()
        sc = _lib.Schedule()
        _lib.check(self._lib.dnsbox_autotune(self._h, _ptr(uh), int(nsteps), ctypes.byref(sc)))
        return self._sched_dict(sc, self.precision == "tc_split")

    def implicit_iterations(self) -> int:
        """Fixed-point iterations of the last semi-implicit step."""
        return self._lib.dnsbox_implicit_iterations(self._h)

    def step_pruned(self) -> bool:
        """Whether the last step call ran the pruned (2/3-rule) passes."""
        return self._lib.dnsbox_step_pruned(self._h) == 1

    # ------------------------------------------------------- time-horizon gradients
    def heun_step_vjp(self, uh, g):
        """Transpose of one fixed-dt IF-Heun step linearised at uh, applied to g."""
        self._check_state(uh)
        g = g.contiguous()
        self._check_state(g, "g")
        out = torch.empty_like(uh)
        self._sync_stream()
        _lib.check(self._lib.dnsbox_heun_step_vjp(self._h, _ptr(uh), _ptr(g), _ptr(out)))
        return out

    def heun_steps_vjp(self, u0, nsteps, gT, every=32, want_uT=False):
        """Transpose of nsteps fixed-dt IF-Heun steps from u0 applied to gT, with
        checkpoints every `every` steps; returns g0 (and u(T) when want_uT)."""
        self._check_state(u0)
        gT = gT.contiguous()
        self._check_state(gT, "gT")
        g0 = torch.empty_like(u0)
        uT = torch.empty_like(u0) if want_uT else None
        self._sync_stream()
        _lib.check(self._lib.dnsbox_heun_steps_vjp(self._h, _ptr(u0), int(nsteps), int(every), _ptr(gT),
                                                   _ptr(g0), _ptr(uT) if uT is not None else None))
        return (g0, uT) if want_uT else g0

    def orbit_residual(self, u0, nsteps, every=32, grad=True):
        """Periodic-orbit residual J = 1/2 <|u(T) - u0|^2> (T = nsteps dt) and,
        with grad, its gradient; returns J or (J, grad)."""
        self._check_state(u0)
        gr = torch.empty_like(u0) if grad else None
        self._sync_stream()
        v = ctypes.c_double()
        _lib.check(self._lib.dnsbox_orbit_residual(self._h, _ptr(u0), int(nsteps), int(every),
                                                   _ptr(gr) if gr is not None else None, ctypes.byref(v)))
        return (v.value, gr) if grad else v.value

    # ---------------------------------------------------------------- transforms
    def c2r(self, spec: torch.Tensor) -> torch.Tensor:
        """Unnormalised 3D C2R of one spectral field (nz, ny, nxh)."""
        assert spec.shape == (self.nz, self.ny, self.nxh) and spec.dtype == self.cdtype and spec.is_contiguous()
        out = torch.empty((self.nz, self.ny, self.nx), dtype=self.rdtype, device=self.device)
        self._sync_stream()
        _lib.check(self._lib.dnsbox_c2r(self._h, _ptr(spec), _ptr(out)))
        return out

    def r2c(self, phys: torch.Tensor) -> torch.Tensor:
        """Unnormalised 3D R2C of one physical field (nz, ny, nx)."""
        assert phys.shape == (self.nz, self.ny, self.nx) and phys.dtype == self.rdtype and phys.is_contiguous()
        out = torch.empty((self.nz, self.ny, self.nxh), dtype=self.cdtype, device=self.device)
        self._sync_stream()
        _lib.check(self._lib.dnsbox_r2c(self._h, _ptr(phys), _ptr(out)))
        return out

    # ---------------------------------------------------------------- measurement
    def profile(self, on: bool = True):
        _lib.check(self._lib.dnsbox_profile_enable(self._h, int(on)))

    def profile_read(self, reset: bool = True):
        """Per-pass summed CUDA-event time (ms) and launch counts since the last reset."""
        self._sync_stream()
        pr = _lib.Profile()
        _lib.check(self._lib.dnsbox_profile_read(self._h, ctypes.byref(pr), int(reset)))
        return {"ms": {n: pr.ms[i] for i, n in enumerate(_lib.PASS_NAMES)},
                "launches": {n: int(pr.launches[i]) for i, n in enumerate(_lib.PASS_NAMES)},
                "total_launches": int(pr.total_launches)}

    # ---------------------------------------------------------------- host I/O
    def upload_state(self, host: np.ndarray, uh: torch.Tensor):
        """host: complex128 (3, nxh, ny, nz) -- p3dfft STRIDE1 (kz fastest)."""
        host = np.ascontiguousarray(host, np.complex128)
        assert host.shape == (3, self.nxh, self.ny, self.nz)
        self._check_state(uh)
        self._sync_stream()
        _lib.check(self._lib.dnsbox_upload_state(self._h, ctypes.c_void_p(host.ctypes.data), _ptr(uh)))

    def download_state(self, uh: torch.Tensor, host: np.ndarray | None = None):
        self._check_state(uh)
        if host is None:
            host = np.empty((3, self.nxh, self.ny, self.nz), np.complex128)
        self._sync_stream()
        _lib.check(self._lib.dnsbox_download_state(self._h, _ptr(uh), ctypes.c_void_p(host.ctypes.data)))
        return host

    def upload_physical(self, host: np.ndarray, uh: torch.Tensor):
        """host: float64 (3, nz, ny, nx), x fastest; R2C into uh (state_u2uhat)."""
        host = np.ascontiguousarray(host, np.float64)
        assert host.shape == (3, self.nz, self.ny, self.nx)
        self._check_state(uh)
        self._sync_stream()
        _lib.check(self._lib.dnsbox_upload_physical(self._h, ctypes.c_void_p(host.ctypes.data), _ptr(uh)))

    def download_physical(self, uh: torch.Tensor, host: np.ndarray | None = None):
        """C2R * scalemodes (state_uhat2u) into float64 (3, nz, ny, nx)."""
        self._check_state(uh)
        if host is None:
            host = np.empty((3, self.nz, self.ny, self.nx), np.float64)
        self._sync_stream()
        _lib.check(self._lib.dnsbox_download_physical(self._h, _ptr(uh), ctypes.c_void_p(host.ctypes.data)))
        return host
