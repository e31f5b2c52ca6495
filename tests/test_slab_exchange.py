"""The slab decomposition's layout contract and its all-to-all on two gloo ranks
(CPU): each rank transforms its z-planes (x R2C, y FFT), packs chunk d = ky rows of
rank d times 1/P, exchanges with ``slab_fft.exchange`` (the same call the GPU driver
makes), and transforms the received k-slab along z.  The k-slabs equal the ky rows
of numpy's rfftn / (Nx Ny Nz), and the inverse exchange returns each rank's planes.
torch.fft stands in for the CUDA passes here; the GPU tests check those passes and
the CUDA pack / unpack against the same contract."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from meumapps_ss_b200.slab_fft import exchange, slab_geometry

SHAPE = (16, 24, 32)  # (Nx, Ny, Nz)


def _field():
    nx, ny, nz = SHAPE
    return np.random.default_rng(5).standard_normal((nz, ny, nx))


def _rank(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        nx, ny, nz = SHAPE
        g = slab_geometry(nx, ny, nz, world)
        nzl, nyl, nxh, P = g["nzl"], g["nyl"], g["nxh"], g["P"]
        x = _field()
        mine = torch.tensor(x[rank * nzl:(rank + 1) * nzl])
        planes = torch.fft.fft(torch.fft.rfft(mine, dim=2), dim=1)  # [z][ky][kx]
        send = (planes.reshape(nzl, P, nyl, nxh).permute(1, 0, 2, 3) / P).contiguous()
        kslab = torch.empty((P, nzl, nyl, nxh), dtype=send.dtype)
        exchange(send, kslab)
        k = torch.fft.fft(kslab.reshape(nz, nyl, nxh), dim=0) / (nx * nyl * nz)
        ref = np.fft.rfftn(x, axes=(0, 1, 2)) / (nx * ny * nz)
        err_f = float(np.max(np.abs(k.numpy() - ref[:, rank * nyl:(rank + 1) * nyl])))
        # inverse: z iFFT, chunk d of the k-slab to rank d, unpack into ky rows, y iFFT, x C2R
        kz = torch.fft.ifft(k, dim=0) * nz
        recv = torch.empty((P, nzl, nyl, nxh), dtype=kz.dtype)
        exchange(kz.reshape(P, nzl, nyl, nxh).contiguous(), recv)
        pl = recv.permute(1, 0, 2, 3).reshape(nzl, ny, nxh)
        back = torch.fft.irfft(torch.fft.ifft(pl, dim=1) * ny, n=nx, dim=2) * nx
        err_b = float(np.max(np.abs(back.numpy() - x[rank * nzl:(rank + 1) * nzl])))
        q.put((rank, err_f, err_b))
    finally:
        dist.destroy_process_group()


def test_slab_contract_two_gloo_ranks():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get() for _ in range(2))
    for rank, ef, eb in res:
        assert ef < 1e-13, (rank, ef)
        assert eb < 1e-12, (rank, eb)


def test_geometry_rules():
    assert slab_geometry(32, 48, 64, 4) == {"nzl": 16, "nyl": 12, "nxh": 17, "P": 4}
    try:
        slab_geometry(32, 48, 64, 5)
    except ValueError:
        pass
    else:
        raise AssertionError("5 ranks accepted")
