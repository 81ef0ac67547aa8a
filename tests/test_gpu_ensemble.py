"""Batched boxes and ensembles (96 boxes of 32^3, 64^3 and 96^3 with their own seeds and viscosities) against single-box runs."""
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


def test_config2_96_boxes_300_steps_against_fp64():
    """Config 2 as specified: 96 boxes (32 each of 32^3, 64^3, 96^3), seeds
    0..95, nu log-uniform in [5e-3, 5e-2] from seed 1000, k0 = 3, dt = 1e-3,
    IF-Heun, FP32 state, 300 steps as CUDA-graph replays; every box against
    its own plain FP64 run.  Bars: velocity relative L2 <= 1e-5, kinetic
    energy and dissipation of the last step <= 1e-5 relative (FP32 storage;
    decaying turbulence at these viscosities is not chaotic enough to
    amplify round-off over 0.3 time units)."""
    from dnsbox_b200.ensemble import Ensemble, config2_nus, make_group
    ns = 300
    nus = config2_nus(96, seed=1000)
    groups = []
    for gi, n in enumerate((32, 64, 96)):
        sl = slice(32 * gi, 32 * (gi + 1))
        groups.append((n, make_group(n, 32, seeds=range(32 * gi, 32 * (gi + 1)), nus=nus[sl], dt=1e-3), sl))
    ens = Ensemble([g for _, g, _ in groups])
    ens.run(ns - 1)                 # create() already advanced one step
    torch.cuda.synchronize()
    worst = {"vel": 0.0, "ekin": 0.0, "diss": 0.0}
    for n, (gb, gu), sl in groups:
        last = gb.diag_read(1)[0]
        for b, (nu, sd) in enumerate(zip(nus[sl], range(sl.start, sl.stop))):
            s, us = _single(n, float(nu), sd, "fp64", bandlim=False, tstep_fix=True, dt=1e-3)
            recs = s.step(us, ns)
            worst["vel"] = max(worst["vel"], rel(gu[:, b].to(torch.complex128), us))
            worst["ekin"] = max(worst["ekin"], abs(last[b]["ekin"] - recs[-1]["ekin"]) / recs[-1]["ekin"])
            worst["diss"] = max(worst["diss"], abs(last[b]["dissipation"] - recs[-1]["dissipation"])
                                / recs[-1]["dissipation"])
            s.close()
    ens.close()
    print("config 2, 96 boxes x 300 steps, FP32 ensemble vs FP64 singles:", worst)
    assert worst["vel"] < 1e-5 and worst["ekin"] < 1e-5 and worst["diss"] < 1e-5


def test_sharded_config2_equals_unsharded():
    """The config-2 ensemble split as over two ranks (each share run here in
    turn on one GPU, in its own captured graph) advances every box exactly as
    the whole 96-box ensemble does, bit for bit: sharding changes which boxes
    share a launch, not the per-box arithmetic."""
    from dnsbox_b200.ensemble import Ensemble, config2_local
    ns = 3
    whole = config2_local(0, 1)
    ens = Ensemble([bu for _, _, bu in whole])
    ens.run(ns)
    torch.cuda.synchronize()
    ref = {gi: u[:, j].cpu() for _, idx, (_, u) in whole for j, gi in enumerate(idx)}
    ens.close()
    seen = set()
    for rank in range(2):
        part = config2_local(rank, 2)
        e = Ensemble([bu for _, _, bu in part])
        e.run(ns)
        torch.cuda.synchronize()
        for _, idx, (box, u) in part:
            for j, gi in enumerate(idx):
                got = (u[:, j] if box.nbatch > 1 else u).cpu()
                assert torch.equal(got, ref[gi])
                seen.add(gi)
        e.close()
    assert seen == set(range(96))


@pytest.mark.parametrize("n,prec", [(32, "fp64"), (48, "fp32"), (96, "fp32"), (128, "tc_split")])
def test_batched_pruned_passes_equal_full_passes(n, prec):
    """A batched context prunes the 2/3-rule zeros as a single box does: with
    per-box CFL control and forcing, the pruned steps equal the full ones bit
    for bit (states and step records)."""
    from dnsbox_b200.ops import Box
    nb, ns = 3, 4
    nus = [2e-3, 4e-3, 8e-3]
    kw = dict(kCutOff=2.5, Pin=0.1, bandlim=True, courant_min=0.5, courant_max=0.5, dt_max=1e-2, dt=1e-3)
    out = []
    for prune in (True, False):
        box = Box(n, nbatch=nb, nu=nus[0], precision=prec, prune=prune, **kw)
        box.set_batch_nu(nus)
        u = box.zeros()
        for b in range(nb):
            u[:, b] = box.from_numpy(ic.random_field(n, seed=20 + b, k0=3.0))
        recs = box.step(u, ns)
        out.append((u.cpu(), recs, box.step_pruned()))
        box.close()
    (up, rp, pp), (uf, rf, pf) = out
    assert pp and not pf
    assert torch.equal(up, uf)
    for i in range(ns):
        for b in range(nb):
            assert rp[i][b]["ekin"] == rf[i][b]["ekin"] and rp[i][b]["dt"] == rf[i][b]["dt"]


def test_ensemble_pruned_graph_and_full_fallback():
    """The ensemble replays the pruned graph while every state vanishes on its
    cut set, and the full graph once a state has content there; both equal the
    eager steps of the same contexts bit for bit."""
    from dnsbox_b200.ensemble import Ensemble, config2_nus, make_group
    spec = [(16, 2), (32, 3)]
    groups, eager = [], []
    for gi, (n, nb) in enumerate(spec):
        nus = config2_nus(nb, seed=2000 + n)
        groups.append(make_group(n, nb, seeds=range(10 * gi, 10 * gi + nb), nus=nus, dt=1e-3))
        eager.append(make_group(n, nb, seeds=range(10 * gi, 10 * gi + nb), nus=nus, dt=1e-3))
    ens = Ensemble(groups)
    ens.run(2)
    assert ens.pruned()
    for box, u in eager:
        box.step(u, 3, diag=False)
        assert box.step_pruned()
    torch.cuda.synchronize()
    for (gb, gu), (eb, eu) in zip(groups, eager):
        assert torch.equal(gu, eu)
    # content on the cut set of one box (kz = 12 of n = 32 lies past the 2/3 cut)
    for _, u in (groups[1], eager[1]):
        u[0, 1, 12, 0, 0] = 1e-3
    ens.run(2)
    assert not ens.pruned()
    eager[1][0].step(eager[1][1], 2, diag=False)
    assert not eager[1][0].step_pruned()
    eager[0][0].step(eager[0][1], 2, diag=False)
    torch.cuda.synchronize()
    for (gb, gu), (eb, eu) in zip(groups, eager):
        assert torch.equal(gu, eu)
    ens.close()
