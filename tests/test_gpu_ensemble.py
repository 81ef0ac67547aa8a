"""Batched boxes and ensembles (SURVEY config 2) against single-box runs."""
import numpy as np
import pytest
import torch

from dnsbox_b200 import ic

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float((a - b).abs().norm() / b.abs().norm())


def _single(n, nu, seed, precision="fp64", **kw):
    from dnsbox_b200.ops import Box
    b = Box(n, precision=precision, nu=nu, **kw)
    return b, b.from_numpy(ic.random_field(n, seed=seed, k0=3.0))


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_batched_box_equals_single_boxes_fixed_dt(prec):
    from dnsbox_b200.ensemble import make_group
    n, nb, ns = 24, 4, 8
    nus = [0.005, 0.01, 0.02, 0.04]
    box, u = make_group(n, nb, seeds=range(nb), nus=nus, dt=2e-3, precision=prec)
    recs = box.step(u, ns)
    for b in range(nb):
        s, us = _single(n, nus[b], b, prec, bandlim=False, tstep_fix=True, dt=2e-3)
        r1 = s.step(us, ns)
        assert rel(u[:, b], us) < 1e-14
        assert abs(recs[-1][b]["ekin"] - r1[-1]["ekin"]) <= 1e-14 * r1[-1]["ekin"]
        assert abs(recs[-1][b]["dissipation"] - r1[-1]["dissipation"]) <= 1e-13 * r1[-1]["dissipation"]


def test_batched_box_per_box_cfl_and_forcing():
    from dnsbox_b200.ops import Box
    n, nb, ns = 32, 3, 5
    nus = [2e-3, 4e-3, 8e-3]
    kw = dict(kCutOff=2.5, Pin=0.1, bandlim=True, courant_min=0.5, courant_max=0.5, dt_max=1e-2, dt=1e-3)
    box = Box(n, nbatch=nb, nu=nus[0], **kw)
    box.set_batch_nu(nus)
    u = box.zeros()
    for b in range(nb):
        u[:, b] = box.from_numpy(ic.random_field(n, seed=10 + b, k0=3.0))
    recs = box.step(u, ns)
    for b in range(nb):
        s, us = _single(n, nus[b], 10 + b, **kw)
        r1 = s.step(us, ns)
        assert rel(u[:, b], us) < 1e-14
        for i in range(ns):
            assert recs[i][b]["dt"] == r1[i]["dt"]
            assert recs[i][b]["courant"] == r1[i]["courant"]
            assert recs[i][b]["eband"] == r1[i]["eband"]


def test_ensemble_graph_equals_eager_and_fp64_runs():
    """Mixed sizes in one graph per step; every FP32 box against its own FP64 run."""
    from dnsbox_b200.ensemble import Ensemble, config2_nus, make_group
    spec = [(16, 3), (24, 2), (32, 2)]
    ns = 12
    groups, eager = [], []
    seed = 0
    for n, nb in spec:
        nus = config2_nus(nb, seed=1000 + n)
        g = make_group(n, nb, seeds=range(seed, seed + nb), nus=nus, dt=1e-3)
        e = make_group(n, nb, seeds=range(seed, seed + nb), nus=nus, dt=1e-3)
        groups.append((g, nus, list(range(seed, seed + nb))))
        eager.append(e)
        seed += nb
    ens = Ensemble([g for g, _, _ in groups])
    ens.run(ns - 1)                 # create() already advanced one step
    torch.cuda.synchronize()
    for (box, u), _ in zip(eager, groups):
        box.step(u, ns, diag=False)
    for ((gb, gu), nus, seeds), (eb, eu) in zip(groups, eager):
        assert torch.equal(gu, eu)                       # graph replay is bitwise the eager step
        rg = gb.diag_read(ns)
        re_ = eb.diag_read(ns)
        assert [r["ekin"] for r in rg[-1]] == [r["ekin"] for r in re_[-1]]
        for b, (nu, sd) in enumerate(zip(nus, seeds)):
            s, us = _single(gb.nx, float(nu), sd, "fp64", bandlim=False, tstep_fix=True, dt=1e-3)
            s.step(us, ns, diag=False)
            assert rel(gu[:, b].to(torch.complex128), us) < 1e-5
    ens.close()
