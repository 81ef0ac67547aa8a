"""The slab-decomposed transform (dnsbox_slab_*, p3dfft's 1 x P
decomposition of variables.f90:131-157) on one GPU: P ranks are emulated in
one process, each with its own slab object and buffers, and the all-to-all
between the local halves is done by device copies (no kernel waits on
another).  The assembled spectrum is checked against the oracle's R2C
(pocketfft) and the library's single-box dnsbox_r2c, the inverse against the
physical field; then the same transform runs through torch.distributed's NCCL
all-to-all on a one-rank process group."""
import datetime
import socket

import numpy as np
import pytest
import torch

from oracle import dnsbox_oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def _emulate(slabs, send_fn, finish_fn):
    """Local halves on every rank, block exchange by copies, finishing halves."""
    for s in slabs:
        send_fn(s)
    p = len(slabs)
    for q in range(p):
        for r in range(p):
            slabs[q].recv[r].copy_(slabs[r].send[q])
    return [finish_fn(s) for s in slabs]


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-13), ("fp32", 8e-7)])
@pytest.mark.parametrize("shape,p", [((32, 48, 64), 1), ((32, 48, 64), 2), ((32, 48, 64), 4),
                                     ((64, 32, 16), 8), ((24, 96, 48), 3)])
def test_slab_transforms_match_the_oracle(prec, tol, shape, p):
    from dnsbox_b200.ops import Box
    from dnsbox_b200.slab import SlabFFT
    nx, ny, nz = shape
    g = O.Grid(O.Params(nx=nx, ny=ny, nz=nz))
    rng = np.random.default_rng(7)
    f = rng.standard_normal((nz, ny, nx))
    want = g.r2c(f)
    slabs = [SlabFFT(nx, ny, nz, precision=prec, rank=r, nranks=p) for r in range(p)]
    rd = slabs[0].rdtype
    phys = [torch.from_numpy(f[s.phys_start[0]:s.phys_start[0] + s.phys_size[0]].copy()).to("cuda", rd)
            for s in slabs]
    specs = [torch.full(s.spec_size, complex("nan"), dtype=s.cdtype, device="cuda") for s in slabs]
    _emulate(slabs, lambda s: s.forward_local(phys[s.rank]), lambda s: s.forward_finish(specs[s.rank]))
    got = torch.cat(specs, dim=1).cpu().numpy()
    assert rel(got, want) < tol
    box = Box(nx=nx, ny=ny, nz=nz, precision=prec)
    lib = box.r2c(torch.from_numpy(f).to("cuda", rd)).cpu().numpy()
    assert rel(got, lib) < tol
    box.close()
    # inverse: the unnormalised C2R of the spectrum is N f
    outs = [torch.full(s.phys_size, float("nan"), dtype=rd, device="cuda") for s in slabs]
    _emulate(slabs, lambda s: s.backward_local(specs[s.rank]), lambda s: s.backward_finish(outs[s.rank]))
    back = torch.cat(outs, dim=0).cpu().numpy()
    assert rel(back, f * (nx * ny * nz)) < tol
    for s in slabs:
        s.close()


def test_slab_rejects_bad_partitions():
    from dnsbox_b200._lib import DnsboxError
    from dnsbox_b200.slab import SlabFFT
    with pytest.raises(DnsboxError):
        SlabFFT(32, 48, 64, rank=0, nranks=5)          # 5 divides neither 48 nor 64
    with pytest.raises(DnsboxError):
        SlabFFT(32, 48, 64, rank=2, nranks=2)
    with pytest.raises(DnsboxError):
        SlabFFT(40, 48, 64, rank=0, nranks=2)          # unsupported length
    s = SlabFFT(32, 48, 64, rank=0, nranks=2)
    with pytest.raises(ValueError):
        s.forward_local(torch.zeros((64, 48, 32), dtype=torch.float64, device="cuda"))   # the whole box, not the slab
    s.close()


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def test_slab_through_nccl_one_rank():
    import torch.distributed as dist
    from dnsbox_b200.slab import SlabFFT
    nx, ny, nz = 32, 32, 64
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        s = SlabFFT(nx, ny, nz, precision="fp64")
        assert (s.rank, s.nranks) == (0, 1)
        g = O.Grid(O.Params(nx=nx, ny=ny, nz=nz))
        f = np.random.default_rng(2).standard_normal((nz, ny, nx))
        spec = s.r2c(torch.from_numpy(f).cuda())
        assert rel(spec.cpu().numpy(), g.r2c(f)) < 1e-13
        back = s.c2r(spec)
        assert rel(back.cpu().numpy(), f * nx * ny * nz) < 1e-13
        torch.cuda.synchronize()
        s.close()
    finally:
        dist.destroy_process_group()


# ---------------------------------------------------------------- rhs_nonlinear over the slabs
def _emulate_rhs(slabs, states, outs):
    """The three halves on every rank with the exchanges and reductions done
    by copies: five and three per-field all-to-alls, the band energy summed and
    the CFL maxima reduced over the ranks."""
    p = len(slabs)
    for s in slabs:
        s.rhs_begin(states[s.rank])
    for f in range(5):
        for q in range(p):
            for r in range(p):
                slabs[q].recv5[f][r].copy_(slabs[r].send5[f][q])
    eb = sum(s.eband.clone() for s in slabs)
    for s in slabs:
        s.eband.copy_(eb)
        s.rhs_middle()
    for f in range(3):
        for q in range(p):
            for r in range(p):
                slabs[q].recv3[f][r].copy_(slabs[r].send3[f][q])
    um = torch.stack([s.umax.clone() for s in slabs]).max(dim=0).values
    for s in slabs:
        s.umax.copy_(um)
        s.rhs_finish(states[s.rank], outs[s.rank])
    return float(eb.item()), um.cpu().numpy()


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 2e-6)])
@pytest.mark.parametrize("shape,p,bandlim", [((32, 32, 32), 2, True), ((32, 48, 64), 4, True),
                                             ((24, 48, 48), 3, False), ((64, 32, 16), 8, True)])
def test_slab_rhs_matches_the_box_and_the_oracle(prec, tol, shape, p, bandlim):
    from dnsbox_b200.ops import Box
    from dnsbox_b200.slab import SlabFFT
    nx, ny, nz = shape
    kw = dict(nu=0.01, kCutOff=2.5, Pin=0.1, bandlim=bandlim)
    g = O.Grid(O.Params(nx=nx, ny=ny, nz=nz, **kw))
    rng = np.random.default_rng(5)
    uh = O.state_dealias(g, O.state_project(g, O.state_u2uhat(g, rng.standard_normal((3, nz, ny, nx)))))
    want = O.rhs_nonlinear(g, uh)
    box = Box(nx=nx, ny=ny, nz=nz, precision=prec, **kw)
    ub = box.from_numpy(uh)
    nb, eb_box = box.rhs_nonlinear(ub)
    umax_box = [float(np.abs(box.c2r(ub[c]).cpu().numpy()).max()) for c in range(3)]
    slabs = [SlabFFT(nx, ny, nz, precision=prec, rank=r, nranks=p) for r in range(p)]
    for s in slabs:
        s.setup_rhs(**kw)
    nyl = ny // p
    states = [ub[:, :, r * nyl:(r + 1) * nyl, :].contiguous() for r in range(p)]
    outs = [torch.full(s.state_shape(), complex("nan"), dtype=s.cdtype, device="cuda") for s in slabs]
    eb, um = _emulate_rhs(slabs, states, outs)
    got = torch.cat(outs, dim=2).cpu().numpy()
    assert rel(got, want) < tol
    assert rel(got, nb.cpu().numpy()) < tol
    if bandlim:
        assert abs(eb - eb_box) <= (1e-12 if prec == "fp64" else 1e-6) * abs(eb_box)
    # CFL maxima: max |u_i| of the physical velocity, which the unnormalised C2R
    # of the state gives N^3 times
    s3 = 1.0 / (nx * ny * nz)
    assert np.allclose(um, np.array(umax_box) * s3, rtol=1e-12 if prec == "fp64" else 2e-6)
    for s in slabs:
        s.close()
    box.close()


def test_slab_rhs_through_nccl_one_rank():
    import torch.distributed as dist
    from dnsbox_b200.ops import Box
    from dnsbox_b200.slab import SlabFFT
    n = 32
    kw = dict(nu=0.01, kCutOff=2.5, Pin=0.1, bandlim=True)
    g = O.Grid(O.Params(nx=n, ny=n, nz=n, **kw))
    uh = O.state_dealias(g, O.state_project(g, O.state_u2uhat(g, np.random.default_rng(8).standard_normal((3, n, n, n)))))
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        s = SlabFFT(n, n, n, precision="fp64")
        s.setup_rhs(**kw)
        out, eb, um = s.rhs_nonlinear(torch.from_numpy(uh).cuda())
        assert rel(out.cpu().numpy(), O.rhs_nonlinear(g, uh)) < 1e-12
        box = Box(n, **kw)
        _, eb_box = box.rhs_nonlinear(box.from_numpy(uh))
        assert abs(eb - eb_box) <= 1e-12 * abs(eb_box)
        torch.cuda.synchronize()
        s.close()
        box.close()
    finally:
        dist.destroy_process_group()


# ---------------------------------------------------------------- IF-Heun over the slabs
def _emulate_stage(slabs, states_in, finish):
    p = len(slabs)
    for s in slabs:
        s.rhs_begin(states_in[s.rank])
    for f in range(5):
        for q in range(p):
            for r in range(p):
                slabs[q].recv5[f][r].copy_(slabs[r].send5[f][q])
    eb = sum(s.eband.clone() for s in slabs)
    for s in slabs:
        s.eband.copy_(eb)
        s.rhs_middle()
    for f in range(3):
        for q in range(p):
            for r in range(p):
                slabs[q].recv3[f][r].copy_(slabs[r].send3[f][q])
    for s in slabs:
        finish(s)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 2e-6)])
@pytest.mark.parametrize("shape,p", [((32, 32, 32), 2), ((32, 48, 64), 4)])
def test_slab_heun_steps_match_the_box(prec, tol, shape, p):
    """Three fixed-dt IF-Heun steps (dnsboxheun.f90:88-126, tStepFix) on the
    slabs of P emulated ranks against the single box's dnsbox_step."""
    from dnsbox_b200.ops import Box
    from dnsbox_b200.slab import SlabFFT
    nx, ny, nz = shape
    dt, nsteps = 4e-3, 3
    kw = dict(nu=0.01, kCutOff=2.5, Pin=0.1, bandlim=True)
    g = O.Grid(O.Params(nx=nx, ny=ny, nz=nz, **kw))
    rng = np.random.default_rng(9)
    uh = O.state_dealias(g, O.state_project(g, O.state_u2uhat(g, 0.05 * rng.standard_normal((3, nz, ny, nx)))))
    box = Box(nx=nx, ny=ny, nz=nz, precision=prec, tstep_fix=True, dt=dt, **kw)
    ub = box.from_numpy(uh)
    box.step(ub, nsteps, diag=False)
    want = ub.cpu().numpy()
    slabs = [SlabFFT(nx, ny, nz, precision=prec, rank=r, nranks=p) for r in range(p)]
    for s in slabs:
        s.setup_rhs(**kw)
    nyl = ny // p
    u0 = torch.from_numpy(uh).to("cuda", slabs[0].cdtype)
    us = [u0[:, :, r * nyl:(r + 1) * nyl, :].contiguous() for r in range(p)]
    ustar = [torch.empty_like(u) for u in us]
    for _ in range(nsteps):
        _emulate_stage(slabs, us, lambda s: s.heun_finish(us[s.rank], ustar[s.rank], False, dt))
        _emulate_stage(slabs, ustar, lambda s: s.heun_finish(ustar[s.rank], us[s.rank], True, dt))
    got = torch.cat(us, dim=2).cpu().numpy()
    assert rel(got, want) < tol
    # and the oracle's IF-Heun (FP64 form only: the FP32 state drifts by its rounding)
    if prec == "fp64":
        w = uh
        for _ in range(nsteps):
            w = O.heun_step(g, w, dt)
        assert rel(got, w) < 1e-12
    for s in slabs:
        s.close()
    box.close()


def test_slab_heun_through_nccl_one_rank():
    import torch.distributed as dist
    from dnsbox_b200.ops import Box
    from dnsbox_b200.slab import SlabFFT
    n, dt = 32, 4e-3
    kw = dict(nu=0.01, kCutOff=2.5, Pin=0.1, bandlim=True)
    g = O.Grid(O.Params(nx=n, ny=n, nz=n, **kw))
    uh = O.state_dealias(g, O.state_project(g, O.state_u2uhat(g, 0.05 * np.random.default_rng(4).standard_normal((3, n, n, n)))))
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        s = SlabFFT(n, n, n, precision="fp64")
        s.setup_rhs(**kw)
        u = torch.from_numpy(uh).cuda()
        recs = s.heun_step(u, dt, 2)
        box = Box(n, tstep_fix=True, dt=dt, **kw)
        ub = box.from_numpy(uh)
        want = box.step(ub, 2)
        assert rel(u.cpu().numpy(), ub.cpu().numpy()) < 1e-12
        for r, w in zip(recs, want):   # the step records, as the single box's
            for k in ("t", "dt", "ekin", "dissipation", "injected_power", "courant", "eband"):
                assert abs(r[k] - w[k]) <= 1e-12 * abs(w[k]), (k, r[k], w[k])
            assert np.allclose(r["umax"], w["umax"], rtol=1e-12)
        torch.cuda.synchronize()
        s.close()
        box.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 2e-6)])
def test_slab_heun_with_courant_control_matches_the_box(prec, tol):
    """CFL-controlled IF-Heun over P = 2 emulated ranks: the step set from the
    reduced CFL maxima of each step's initial state (set_time_step on
    io_Courant) matches the single box's device rule, steps and state."""
    from dnsbox_b200.ops import Box
    from dnsbox_b200.slab import SlabFFT
    nx = ny = nz = 32
    p, dt0, nsteps, cfl = 2, 4e-3, 3, (0.4, 0.6, 0.01)
    kw = dict(nu=0.01, kCutOff=2.5, Pin=0.1, bandlim=True)
    g = O.Grid(O.Params(nx=nx, ny=ny, nz=nz, **kw))
    rng = np.random.default_rng(12)
    uh = O.state_dealias(g, O.state_project(g, O.state_u2uhat(g, 0.05 * rng.standard_normal((3, nz, ny, nx)))))
    box = Box(nx=nx, ny=ny, nz=nz, precision=prec, dt=dt0, courant_min=cfl[0], courant_max=cfl[1], dt_max=cfl[2],
              **kw)
    ub = box.from_numpy(uh)
    recs = box.step(ub, nsteps)
    slabs = [SlabFFT(nx, ny, nz, precision=prec, rank=r, nranks=p) for r in range(p)]
    for s in slabs:
        s.setup_rhs(**kw)
    nyl = ny // p
    u0 = torch.from_numpy(uh).to("cuda", slabs[0].cdtype)
    us = [u0[:, :, r * nyl:(r + 1) * nyl, :].contiguous() for r in range(p)]
    ustar = [torch.empty_like(u) for u in us]
    dt, steps, ekin, diss = dt0, [], [], []
    s2 = (1.0 / (nx * ny * nz)) ** 2
    for i in range(nsteps):
        _emulate_stage(slabs, us, lambda s: None)
        um = torch.stack([s.umax.clone() for s in slabs]).max(dim=0).values
        for s in slabs:
            s.umax.copy_(um)
        dt, _ = slabs[0].courant_dt(dt, *cfl, first=(i == 0))
        steps.append(dt)
        for s in slabs:
            s.heun_finish(us[s.rank], ustar[s.rank], False, dt)
        _emulate_stage(slabs, ustar, lambda s: s.heun_finish(ustar[s.rank], us[s.rank], True, dt))
        ed = sum(s.ed.clone() for s in slabs).tolist()      # the sum over the ranks
        ekin.append(ed[0] * s2)
        diss.append(kw["nu"] * ed[1] * s2)
    want_steps = [r["dt"] for r in recs]
    assert np.allclose(steps, want_steps, rtol=1e-13 if prec == "fp64" else 1e-6), (steps, want_steps)
    r_tol = 1e-12 if prec == "fp64" else 2e-6
    assert np.allclose(ekin, [r["ekin"] for r in recs], rtol=r_tol)
    assert np.allclose(diss, [r["dissipation"] for r in recs], rtol=r_tol)
    got = torch.cat(us, dim=2).cpu().numpy()
    assert rel(got, ub.cpu().numpy()) < tol
    for s in slabs:
        s.close()
    box.close()
