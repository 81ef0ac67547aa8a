"""Slab-decomposed 3D FFT over ranks, one GPU each (``dnsbox_slab_*``).

The reference distributes a box with p3dfft's one-dimensional decomposition
(variables.f90:131-157, processor grid 1 x nproc): physical fields in slabs of
nz/P z-planes, spectral fields in slabs of ny/P ky rows, and one MPI all-to-all
inside every p3dfft_ftran_r2c / p3dfft_btran_c2r (dnsbox.f90:44-46, 229-231).
``SlabFFT`` is that transform on B200s: the library runs the local passes on
this rank's GPU and the exchange between them is one all-to-all of P equal
blocks, NCCL over NVLink through ``torch.distributed``.

Layouts (row-major, innermost last):

* physical slab ``(nz/P, ny, nx)`` real, planes ``[rank nz/P, (rank+1) nz/P)``;
* spectral slab ``(nz, ny/P, nx/2+1)`` complex, ky rows ``[rank ny/P, ...)``.

Transforms are unnormalised, as ``Box.r2c`` / ``Box.c2r`` and p3dfft's.

``SlabFFT.rhs_nonlinear`` is the reference's ``rhs_nonlinear`` (rhs.f90:18-135)
on a spectral ky-slab state ``(3, nz, ny/P, nx/2+1)``: the single-box passes
with eight all-to-alls (five fields out of the inverse z pass, three into the
forward z pass), the band energy summed and the CFL maxima reduced over the
ranks.
"""
from __future__ import annotations

import ctypes
import math

import torch

from . import _lib
from .ops import PRECISION


def slab_extents(nx: int, ny: int, nz: int, nranks: int, rank: int) -> dict:
    """(z, y, x) starts and sizes of a rank's physical and spectral slabs
    (p3dfft_get_dims, 0-based) and the complex elements of one exchange block."""
    if nranks < 1 or not 0 <= rank < nranks:
        raise ValueError(f"rank {rank} of {nranks}")
    if ny % nranks or nz % nranks:
        raise ValueError(f"{nranks} ranks do not divide ny = {ny} and nz = {nz}")
    nzl, nyl, nxh = nz // nranks, ny // nranks, nx // 2 + 1
    return {"phys_start": (rank * nzl, 0, 0), "phys_size": (nzl, ny, nx),
            "spec_start": (0, rank * nyl, 0), "spec_size": (nz, nyl, nxh),
            "block_elems": nzl * nyl * nxh}


def all_reduce(t: torch.Tensor, op: str, group=None) -> None:
    """Sum ("sum") or maximum ("max") of ``t`` over the ranks, in place
    (nothing without a process group)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return
    dist.all_reduce(t, op=dist.ReduceOp.SUM if op == "sum" else dist.ReduceOp.MAX, group=group)


def all_to_all(send: torch.Tensor, recv: torch.Tensor, group=None) -> None:
    """Block q of this rank's ``send`` to rank q, arriving as block r of its
    ``recv`` for sender r (P equal blocks along dim 0).  Without a process
    group: a copy."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        recv.copy_(send)
        return
    s = torch.view_as_real(send) if send.is_complex() else send
    r = torch.view_as_real(recv) if recv.is_complex() else recv
    dist.all_to_all_single(r.reshape(-1), s.reshape(-1), group=group)


class SlabFFT:
    """This rank's part of a slab-decomposed (nx, ny, nz) transform.

    ``rank`` / ``nranks`` default to the process group's; ``exchange`` (default
    :func:`all_to_all` over ``group``) moves the blocks between the local
    halves.  ``r2c`` / ``c2r`` run local half, exchange, finishing half on
    torch's current stream."""

    def __init__(self, nx: int, ny: int, nz: int, precision: str = "fp64", group=None, rank=None, nranks=None,
                 device=None, exchange=None):
        import torch.distributed as dist
        dist_on = dist.is_available() and dist.is_initialized()
        self.rank = int(rank) if rank is not None else (dist.get_rank(group) if dist_on else 0)
        self.nranks = int(nranks) if nranks is not None else (dist.get_world_size(group) if dist_on else 1)
        if precision not in ("fp64", "fp32"):
            raise ValueError("precision must be 'fp64' or 'fp32'")
        self.nx, self.ny, self.nz, self.precision = nx, ny, nz, precision
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else int(device))
        self.rdtype = torch.float64 if precision == "fp64" else torch.float32
        self.cdtype = torch.complex128 if precision == "fp64" else torch.complex64
        self._lib = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(self._lib.dnsbox_slab_create(nx, ny, nz, self.nranks, self.rank, PRECISION[precision],
                                                self.device.index, ctypes.byref(h)))
        self._h = h
        ps, pz, ss, sz = ((ctypes.c_int * 3)() for _ in range(4))
        blk = ctypes.c_size_t()
        _lib.check(self._lib.dnsbox_slab_dims(self._h, ps, pz, ss, sz, ctypes.byref(blk)))
        self.phys_start, self.phys_size = tuple(ps), tuple(pz)
        self.spec_start, self.spec_size = tuple(ss), tuple(sz)
        self.block_elems = blk.value
        self.send = torch.empty((self.nranks, self.block_elems), dtype=self.cdtype, device=self.device)
        self.recv = torch.empty_like(self.send)
        self._group = group
        self._exchange = exchange if exchange is not None else (lambda s, r: all_to_all(s, r, group))

    # -- the halves (the exchange between them is the caller's in these) --
    def _stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _check(self, t: torch.Tensor, shape, dtype, what: str):
        if t.device != self.device or t.dtype != dtype or tuple(t.shape) != tuple(shape) or not t.is_contiguous():
            raise ValueError(f"{what}: expected contiguous {dtype} {tuple(shape)} on {self.device}, "
                             f"got {t.dtype} {tuple(t.shape)} on {t.device}")

    def forward_local(self, phys: torch.Tensor) -> None:
        self._check(phys, self.phys_size, self.rdtype, "physical slab")
        _lib.check(self._lib.dnsbox_slab_ftran_local(self._h, ctypes.c_void_p(phys.data_ptr()),
                                                     ctypes.c_void_p(self.send.data_ptr()), self._stream()))

    def forward_finish(self, spec: torch.Tensor) -> None:
        self._check(spec, self.spec_size, self.cdtype, "spectral slab")
        _lib.check(self._lib.dnsbox_slab_ftran_finish(self._h, ctypes.c_void_p(self.recv.data_ptr()),
                                                      ctypes.c_void_p(spec.data_ptr()), self._stream()))

    def backward_local(self, spec: torch.Tensor) -> None:
        self._check(spec, self.spec_size, self.cdtype, "spectral slab")
        _lib.check(self._lib.dnsbox_slab_btran_local(self._h, ctypes.c_void_p(spec.data_ptr()),
                                                     ctypes.c_void_p(self.send.data_ptr()), self._stream()))

    def backward_finish(self, phys: torch.Tensor) -> None:
        self._check(phys, self.phys_size, self.rdtype, "physical slab")
        _lib.check(self._lib.dnsbox_slab_btran_finish(self._h, ctypes.c_void_p(self.recv.data_ptr()),
                                                      ctypes.c_void_p(phys.data_ptr()), self._stream()))

    # -- whole transforms (p3dfft_ftran_r2c / p3dfft_btran_c2r) --
    def r2c(self, phys: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        spec = out if out is not None else torch.empty(self.spec_size, dtype=self.cdtype, device=self.device)
        self.forward_local(phys)
        self._exchange(self.send, self.recv)
        self.forward_finish(spec)
        return spec

    def c2r(self, spec: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        phys = out if out is not None else torch.empty(self.phys_size, dtype=self.rdtype, device=self.device)
        self.backward_local(spec)
        self._exchange(self.send, self.recv)
        self.backward_finish(phys)
        return phys

    # -- rhs_nonlinear over the slabs --
    def setup_rhs(self, nu: float = 0.0, Q: float = 0.0, kCutOff: float = 2.5, Pin: float = 0.0,
                  bandlim: bool = False, spherical: bool = False, alpha=(1.0, 1.0, 1.0), reduce=None):
        """Physics of the right-hand side (as ``Box``); ``reduce(t, op)``
        (default :func:`all_reduce` over the group) sums the band energy and
        takes the maximum of the CFL maxima over the ranks."""
        p = _lib.Params()
        self._lib.dnsbox_default_params(ctypes.byref(p))
        p.nx, p.ny, p.nz = self.nx, self.ny, self.nz
        p.precision = PRECISION[self.precision]
        p.device = self.device.index
        p.bandlim, p.spherical = int(bandlim), int(spherical)
        p.alpha_x, p.alpha_y, p.alpha_z = alpha
        p.nu, p.Q, p.kCutOff, p.Pin = nu, Q, kCutOff, Pin
        _lib.check(self._lib.dnsbox_slab_rhs_setup(self._h, ctypes.byref(p)))
        shape = (self.nranks, self.block_elems)
        self.send5 = torch.empty((5,) + shape, dtype=self.cdtype, device=self.device)
        self.recv5 = torch.empty_like(self.send5)
        self.send3 = torch.empty((3,) + shape, dtype=self.cdtype, device=self.device)
        self.recv3 = torch.empty_like(self.send3)
        self.eband = torch.zeros(1, dtype=torch.float64, device=self.device)
        self.ed = torch.zeros(2, dtype=torch.float64, device=self.device)
        self._alpha = tuple(float(a) for a in alpha)
        self._phys = dict(nu=float(nu), Q=float(Q), Pin=float(Pin), bandlim=bool(bandlim))
        self._cfl_done = False
        self.t = 0.0
        self.umax = torch.zeros(3, dtype=torch.float64, device=self.device)
        self._reduce = reduce if reduce is not None else (lambda t, op: all_reduce(t, op, self._group))

    def state_shape(self):
        """The spectral ky-slab state: (3, nz, ny/P, nx/2+1)."""
        return (3,) + self.spec_size

    def rhs_begin(self, uh: torch.Tensor) -> None:
        self._check(uh, self.state_shape(), self.cdtype, "state slab")
        _lib.check(self._lib.dnsbox_slab_rhs_begin(self._h, ctypes.c_void_p(uh.data_ptr()),
                                                   ctypes.c_void_p(self.eband.data_ptr()),
                                                   ctypes.c_void_p(self.send5.data_ptr()), self._stream()))

    def rhs_middle(self) -> None:
        _lib.check(self._lib.dnsbox_slab_rhs_middle(self._h, ctypes.c_void_p(self.recv5.data_ptr()),
                                                    ctypes.c_void_p(self.umax.data_ptr()),
                                                    ctypes.c_void_p(self.send3.data_ptr()), self._stream()))

    def rhs_finish(self, uh: torch.Tensor, out: torch.Tensor) -> None:
        self._check(out, self.state_shape(), self.cdtype, "output slab")
        _lib.check(self._lib.dnsbox_slab_rhs_finish(self._h, ctypes.c_void_p(self.recv3.data_ptr()),
                                                    ctypes.c_void_p(uh.data_ptr()),
                                                    ctypes.c_void_p(self.eband.data_ptr()),
                                                    ctypes.c_void_p(out.data_ptr()), self._stream()))

    def _exchange_rhs(self, uh: torch.Tensor) -> None:
        self.rhs_begin(uh)
        for f in range(5):
            self._exchange(self.send5[f], self.recv5[f])
        self._reduce(self.eband, "sum")
        self.rhs_middle()
        for f in range(3):
            self._exchange(self.send3[f], self.recv3[f])
        self._reduce(self.umax, "max")

    def heun_finish(self, uin: torch.Tensor, out: torch.Tensor, corrector: bool, dt: float) -> None:
        """The predictor's (u* into out) or the corrector's (out = u, in place)
        finish; the corrector leaves this rank's (E, D) sums in ``self.ed``."""
        self._check(out, self.state_shape(), self.cdtype, "state slab")
        ed = ctypes.c_void_p(self.ed.data_ptr()) if corrector else None
        _lib.check(self._lib.dnsbox_slab_heun_finish(self._h, ctypes.c_void_p(self.recv3.data_ptr()),
                                                     ctypes.c_void_p(uin.data_ptr()),
                                                     ctypes.c_void_p(self.eband.data_ptr()), int(bool(corrector)),
                                                     float(dt), ctypes.c_void_p(out.data_ptr()), ed, self._stream()))

    def step_record(self, dt: float, courant: float) -> dict:
        """The step record (the Ekin.dat quantities, io.f90:651-658) from the
        corrector's (E, D) sums once they are summed over the ranks."""
        s2 = (1.0 / (self.nx * self.ny * self.nz)) ** 2
        e, d = self.ed.tolist()
        ph = self._phys
        ekin = e * s2
        return {"t": self.t, "dt": dt, "ekin": ekin, "dissipation": ph["nu"] * d * s2,
                "production_literal": 2.0 * ph["Q"] * ekin,
                "injected_power": (ph["Pin"] if ph["bandlim"] else 0.0) + 2.0 * ph["Q"] * ekin,
                "courant": courant, "umax": tuple(self.umax.tolist()), "eband": float(self.eband.item())}

    def courant_number(self, dt: float) -> float:
        """io_Courant (io.f90:664-676) of the reduced CFL maxima."""
        dx = (2.0 * math.pi / self._alpha[0]) / self.nx
        dy = (2.0 * math.pi / self._alpha[1]) / self.ny
        dz = (2.0 * math.pi / self._alpha[2]) / self.nz
        um = self.umax.tolist()
        return um[0] * dt / dx + um[1] * dt / dy + um[2] * dt / dz

    def courant_dt(self, dt: float, courant_min: float, courant_max: float, dt_max: float, first: bool):
        """set_time_step (dnsboxheun.f90:227-246) on io_Courant (io.f90:664-676)
        of the reduced CFL maxima, as the single box's device rule: returns the
        step and its Courant number."""
        c = self.courant_number(dt)
        if first or c > courant_max or (c < courant_min and dt < dt_max):
            nd = ((courant_max + courant_min) / (2.0 * c)) * dt
            if nd > dt_max:
                nd = dt_max
            c = c * nd / dt
            dt = nd
        return dt, c

    def heun_step(self, uh: torch.Tensor, dt: float, nsteps: int = 1, courant=None) -> list:
        """IF-Heun (dnsboxheun.f90:88-126) on this rank's ky slab, in place:
        u* = IF (u + dt N(u)), then u <- (IF u + u*) / 2 + dt/2 N(u*).  With
        ``courant = (courant_min, courant_max, dt_max)`` the step is set from
        the Courant number of each step's initial state (the first step always
        adjusts it, as the reference's first call does), else ``dt`` is fixed
        (tStepFix).  Returns the step records (t after the step, dt, Ekin,
        dissipation, production, Courant number, CFL maxima, band energy)."""
        self._check(uh, self.state_shape(), self.cdtype, "state slab")
        ustar = torch.empty_like(uh)
        recs = []
        for i in range(int(nsteps)):
            self._exchange_rhs(uh)
            eband, umax = float(self.eband.item()), tuple(self.umax.tolist())
            if courant is not None:
                dt, c = self.courant_dt(dt, *courant, first=(i == 0 and not self._cfl_done))
                self._cfl_done = True
            else:
                c = self.courant_number(dt)
            self.heun_finish(uh, ustar, False, dt)
            self._exchange_rhs(ustar)
            self.heun_finish(ustar, uh, True, dt)
            self._reduce(self.ed, "sum")
            self.t += dt
            rec = self.step_record(dt, c)
            rec.update(eband=eband, umax=umax)   # of the step's initial state, as the single box's records
            recs.append(rec)
        return recs

    def rhs_nonlinear(self, uh: torch.Tensor, out: torch.Tensor | None = None):
        """N(u) of this rank's ky slab; returns (N, band energy, (max|u|, max|v|,
        max|w|)), the last two over the whole box."""
        if out is None:
            out = torch.empty(self.state_shape(), dtype=self.cdtype, device=self.device)
        self._exchange_rhs(uh)
        self.rhs_finish(uh, out)
        return out, float(self.eband.item()), tuple(float(v) for v in self.umax.tolist())

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.dnsbox_slab_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
