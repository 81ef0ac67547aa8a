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
