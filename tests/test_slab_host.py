"""Host side of the slab-decomposed transform (dnsbox_b200/slab.py): the
partition of p3dfft's 1 x P processor grid (variables.f90:131-157), the
all-to-all of equal blocks and the sum and max all-reduces on gloo ranks (world size 2 and 3), and a NumPy
model of the decomposition's block layout, which the CUDA halves follow: the
received blocks of a forward transform, in rank order, are the local ky rows
of every z-plane.  No GPU is touched."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from dnsbox_b200.slab import all_reduce, all_to_all, slab_extents


def test_extents_tile_the_grid():
    for nx, ny, nz, p in [(32, 48, 64, 1), (32, 48, 64, 2), (32, 48, 64, 4), (16, 24, 24, 3), (8, 8, 8, 8)]:
        ext = [slab_extents(nx, ny, nz, p, r) for r in range(p)]
        zs = [(e["phys_start"][0], e["phys_size"][0]) for e in ext]
        ys = [(e["spec_start"][1], e["spec_size"][1]) for e in ext]
        assert [z0 for z0, _ in zs] == [r * (nz // p) for r in range(p)] and sum(n for _, n in zs) == nz
        assert [y0 for y0, _ in ys] == [r * (ny // p) for r in range(p)] and sum(n for _, n in ys) == ny
        for e in ext:
            assert e["phys_size"][1:] == (ny, nx) and e["spec_size"][0] == nz and e["spec_size"][2] == nx // 2 + 1
            assert e["block_elems"] == (nz // p) * (ny // p) * (nx // 2 + 1)
    with pytest.raises(ValueError):
        slab_extents(16, 24, 20, 3, 0)
    with pytest.raises(ValueError):
        slab_extents(16, 24, 24, 3, 3)


# --- the block layout, modelled in NumPy (forward: x R2C, y FFT, pack by
# destination; exchange; z FFT of the received blocks as they lie) ---
def _ftran_local(f, p):
    nzl, ny, nx = f.shape
    a = np.fft.fft(np.fft.rfft(f, axis=2), axis=1)            # (nzl, ny, nxh)
    nyl = ny // p
    return np.stack([a[:, q * nyl:(q + 1) * nyl, :].reshape(-1) for q in range(p)])


def _btran_finish(recv, nzl, ny, nx, p):
    nyl, nxh = ny // p, nx // 2 + 1
    planes = np.concatenate([recv[r].reshape(nzl, nyl, nxh) for r in range(p)], axis=1)
    return np.fft.irfft(np.fft.ifft(planes, axis=1) * ny, n=nx, axis=2) * nx


def _exchange(sends):
    p = len(sends)
    return [np.stack([sends[r][q] for r in range(p)]) for q in range(p)]


@pytest.mark.parametrize("p", [1, 2, 4])
def test_numpy_model_of_the_decomposition(p):
    nx, ny, nz = 16, 24, 32
    rng = np.random.default_rng(3)
    f = rng.standard_normal((nz, ny, nx))
    want = np.fft.rfftn(f, axes=(0, 1, 2))
    ext = [slab_extents(nx, ny, nz, p, r) for r in range(p)]
    sends = [_ftran_local(f[e["phys_start"][0]:e["phys_start"][0] + e["phys_size"][0]], p) for e in ext]
    recvs = _exchange(sends)
    for r, e in enumerate(ext):
        spec = np.fft.fft(recvs[r].reshape(e["spec_size"]), axis=0)    # blocks in rank order = (nz, nyl, nxh)
        y0, nyl = e["spec_start"][1], e["spec_size"][1]
        assert np.allclose(spec, want[:, y0:y0 + nyl, :], atol=1e-9)
    # inverse: z FFT into send (block q = planes of rank q), exchange, unpack
    specs = [want[:, e["spec_start"][1]:e["spec_start"][1] + e["spec_size"][1], :] for e in ext]
    sends = [np.fft.ifft(s, axis=0).reshape(p, -1) * nz for s in specs]
    recvs = _exchange(sends)
    for r, e in enumerate(ext):
        z0, nzl = e["phys_start"][0], e["phys_size"][0]
        got = _btran_finish(recvs[r], nzl, ny, nx, p)
        assert np.allclose(got, f[z0:z0 + nzl] * nx * ny * nz, atol=1e-8 * nx * ny * nz)


# --- the exchange on gloo ranks ---
def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        blk = 5
        send = torch.zeros((world, blk), dtype=torch.complex128)
        for d in range(world):
            send[d] = torch.arange(blk) + 1j * (100 * rank + d)    # tagged (sender, destination)
        recv = torch.full_like(send, complex("nan"))
        all_to_all(send, recv)
        ok = all(torch.equal(recv[s], torch.arange(blk) + 1j * (100 * s + rank)) for s in range(world))
        # the band-energy / (E, D) sums and the CFL maxima of the slab stepper
        e = torch.tensor([1.0 + rank], dtype=torch.float64)
        all_reduce(e, "sum")
        m = torch.tensor([float(rank), 10.0 - rank, 0.5], dtype=torch.float64)
        all_reduce(m, "max")
        ok = ok and e.item() == sum(1.0 + r for r in range(world)) and m.tolist() == [world - 1.0, 10.0, 0.5]
        dist.barrier()
        q.put((rank, ok))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_all_to_all_on_gloo_ranks(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert res == [(r, True) for r in range(world)]


def test_all_to_all_single_process_is_a_copy():
    send = torch.arange(12, dtype=torch.float64).reshape(1, 12)
    recv = torch.zeros_like(send)
    all_to_all(send, recv)
    assert torch.equal(send, recv)
