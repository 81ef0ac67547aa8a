"""Ensembles of independent boxes advanced together (one CUDA graph per step).

Boxes of one size share a batched ``Box`` (component-major state
(3, nbox, n, n, n//2+1)); groups of different sizes are captured together by
``dnsbox_ensemble_create``: one replay of the graph advances every box of every
group by one step.  The reference runs one box per MPI job; this serves
parameter sweeps and ensembles of small boxes that would each underfill a GPU.

Across GPUs the boxes shard with no collective on the data path: each rank
advances its contiguous share of every size group (``shard``), and only the
final per-box diagnostics meet on rank 0 (``gather_to_rank0``).
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

    def pruned(self) -> bool:
        """Whether the last run replayed the pruned passes."""
        return self._lib.dnsbox_ensemble_pruned(self._h) == 1

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
        f = torch.from_numpy(ic.random_field(n, seed=int(seed), k0=k0)).to(box.device, box.cdtype)
        if nbox > 1:
            u[:, b] = f
        else:   # a one-box Box has no batch axis
            u.copy_(f)
    return box, u


def config2_nus(nbox: int, seed: int = 1000):
    """nu log-uniform in [5e-3, 5e-2] from a seeded generator."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.exp(rng.uniform(np.log(5e-3), np.log(5e-2), nbox))


def shard(n: int, rank: int, world: int) -> range:
    """This rank's contiguous share of n independent items; shares differ in
    size by at most one and cover 0 .. n-1 once over the ranks."""
    if not (0 <= rank < world):
        raise ValueError(f"rank {rank} outside a world of {world}")
    q, r = divmod(int(n), int(world))
    lo = rank * q + min(rank, r)
    return range(lo, lo + q + (1 if rank < r else 0))


CONFIG2_SIZES = (32, 64, 96)


def config2_local(rank: int = 0, world: int = 1, per_size: int = 32, dt: float = 1e-3, precision: str = "fp32"):
    """This rank's part of the config-2 ensemble: per size in CONFIG2_SIZES its
    share of that group's boxes.  Box g * per_size + i (size group g) keeps its
    global seed and its nu from ``config2_nus(3 * per_size)`` wherever it runs.
    Returns [(n, global indices, (Box, state))] for the non-empty shares."""
    nus = config2_nus(len(CONFIG2_SIZES) * per_size, seed=1000)
    out = []
    for g, n in enumerate(CONFIG2_SIZES):
        idx = [g * per_size + i for i in shard(per_size, rank, world)]
        if idx:
            out.append((n, idx, make_group(n, len(idx), seeds=idx, nus=nus[idx], dt=dt, precision=precision)))
    return out


def gather_to_rank0(local: dict, world: int):
    """{global index: value} of every rank merged on rank 0 (None elsewhere),
    ordered by index; the one collective of a sharded ensemble."""
    import torch.distributed as dist
    if world == 1:
        return dict(sorted(local.items()))
    parts = [None] * world if dist.get_rank() == 0 else None
    dist.gather_object(local, parts, dst=0)
    if dist.get_rank() != 0:
        return None
    merged = {}
    for part in parts:
        for k, v in part.items():
            if k in merged:
                raise ValueError(f"box {k} reported by two ranks")
            merged[k] = v
    return dict(sorted(merged.items()))
