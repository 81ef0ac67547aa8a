"""Ensembles of independent boxes advanced together (one CUDA graph per step).

Boxes of one size share a batched ``Box`` (component-major state
(3, nbox, n, n, n//2+1)); groups of different sizes are captured together by
``dnsbox_ensemble_create``: one replay of the graph advances every box of every
group by one step.  The reference runs one box per MPI job; this serves
parameter sweeps and ensembles of small boxes that would each underfill a GPU.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .ops import Box


class Ensemble:
    def __init__(self, groups):
        """groups: list of (Box, state tensor) pairs; states are advanced in place."""
        self.groups = list(groups)
        lib = _lib.load()
        n = len(self.groups)
        s = torch.cuda.current_stream().cuda_stream
        for box, u in self.groups:
            box._check_state(u)
            _lib.check(lib.dnsbox_set_stream(box._h, ctypes.c_void_p(s)))
        ctxs = (ctypes.c_void_p * n)(*[box._h.value for box, _ in self.groups])
        states = (ctypes.c_void_p * n)(*[u.data_ptr() for _, u in self.groups])
        h = ctypes.c_void_p()
        _lib.check(lib.dnsbox_ensemble_create(ctxs, states, n, ctypes.byref(h)))
        self._h = h
        self._lib = lib

    def run(self, nsteps: int):
        _lib.check(self._lib.dnsbox_ensemble_run(self._h, int(nsteps)))

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.dnsbox_ensemble_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_group(n: int, nbox: int, seeds, nus, k0=3.0, dt=1e-3, precision="fp32", **kw):
    """A batched Box of nbox decaying-turbulence boxes of size n (fixed dt, IF-Heun)
    and its state seeded with ``ic.random_field`` per box."""
    from . import ic
    box = Box(n, precision=precision, nbatch=nbox, nu=float(np.mean(nus)), bandlim=False,
              tstep_fix=True, dt=dt, **kw)
    box.set_batch_nu(nus)
    u = box.zeros()
    for b, seed in enumerate(seeds):
        u[:, b] = torch.from_numpy(ic.random_field(n, seed=int(seed), k0=k0)).to(box.device, box.cdtype)
    return box, u


def config2_nus(nbox: int, seed: int = 1000):
    """nu log-uniform in [5e-3, 5e-2] from a seeded generator."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.exp(rng.uniform(np.log(5e-3), np.log(5e-2), nbox))
