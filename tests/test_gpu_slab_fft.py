"""Slab-decomposed f_trans / inv_trans (meu_slab_fft_*) on the GPU.

* P ranks emulated in one process on one GPU: every rank's planes and columns run
  through the C-ABI on that rank's slab, and the all-to-all is done by copying
  chunk r of rank q's send buffer into slot q of rank r's receive buffer.  The
  gathered k-slabs equal numpy's rfftn / (Nx Ny Nz) and the inverse gives the
  field back, for P = 1, 2, 4 and both precisions (no two ranks' kernels wait on
  one another: the exchange is between launches).
* SlabFFT, the torch.distributed driver, on one rank, with and without an NCCL
  process group.
"""
import ctypes as C

import numpy as np
import pytest

from meumapps_ss_b200 import _lib
from meumapps_ss_b200 import params as P

SHAPE = (32, 48, 64)  # (Nx, Ny, Nz)


def _full(prec, seed=3):
    nx, ny, nz = SHAPE
    rng = np.random.default_rng(seed)
    return rng.standard_normal((nz, ny, nx))


def _tol(prec):
    return 1e-12 if prec == P.PREC_F64 else 3e-6


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [P.PREC_F64, P.PREC_F32])
@pytest.mark.parametrize("nranks", [1, 2, 4])
def test_emulated_ranks_match_numpy(prec, nranks):
    import torch

    L = _lib.lib()
    nx, ny, nz = SHAPE
    nzl, nyl, nxh = nz // nranks, ny // nranks, nx // 2 + 1
    rd = torch.float64 if prec == P.PREC_F64 else torch.float32
    cd = torch.complex128 if prec == P.PREC_F64 else torch.complex64
    x = _full(prec)
    ref = np.fft.rfftn(x, axes=(0, 1, 2)) / (nx * ny * nz)
    hs, sends, reals = [], [], []
    for r in range(nranks):
        h = C.c_void_p()
        assert L.meu_slab_fft_create(nx, ny, nz, nranks, r, prec, C.byref(h)) == 0
        sz = (C.c_int64 * 4)()
        assert L.meu_slab_fft_sizes(h, sz) == 0
        assert list(sz) == [nzl * ny * nx, nzl * nyl * nxh, nz * nyl * nxh, nranks]
        hs.append(h)
        reals.append(torch.tensor(x[r * nzl:(r + 1) * nzl], dtype=rd, device="cuda").contiguous())
        sends.append(torch.empty((nranks, nzl, nyl, nxh), dtype=cd, device="cuda"))
    for r in range(nranks):
        assert L.meu_slab_fft_forward_planes(hs[r], C.c_void_p(reals[r].data_ptr()),
                                             C.c_void_p(sends[r].data_ptr()), None) == 0
    kslabs = []
    for r in range(nranks):
        k = torch.stack([sends[q][r] for q in range(nranks)]).reshape(nz, nyl, nxh).contiguous()
        assert L.meu_slab_fft_forward_columns(hs[r], C.c_void_p(k.data_ptr()), None) == 0
        kslabs.append(k)
    torch.cuda.synchronize()
    got = np.concatenate([k.cpu().numpy() for k in kslabs], axis=1)
    assert np.max(np.abs(got - ref)) <= _tol(prec) * np.max(np.abs(ref))
    # inverse: z iFFT in place, chunk r of rank d's k-slab to rank r, planes
    for r in range(nranks):
        assert L.meu_slab_fft_inverse_columns(hs[r], C.c_void_p(kslabs[r].data_ptr()), None) == 0
    outs = []
    for r in range(nranks):
        recv = torch.stack([kslabs[d].reshape(nranks, nzl, nyl, nxh)[r] for d in range(nranks)]).contiguous()
        out = torch.empty((nzl, ny, nx), dtype=rd, device="cuda")
        assert L.meu_slab_fft_inverse_planes(hs[r], C.c_void_p(recv.data_ptr()), C.c_void_p(out.data_ptr()), None) == 0
        outs.append(out)
    torch.cuda.synchronize()
    back = np.concatenate([o.cpu().numpy() for o in outs], axis=0)
    assert np.max(np.abs(back - x)) <= 10 * _tol(prec) * np.max(np.abs(x))
    for h in hs:
        assert L.meu_slab_fft_launch_count(h) > 0
        L.meu_slab_fft_destroy(h)


@pytest.mark.gpu
def test_slab_fft_rejects_bad_decompositions():
    L = _lib.lib()
    h = C.c_void_p()
    badarg, unsupported = 100, 103  # MEU_ERR_BADARG, MEU_ERR_UNSUPPORTED
    assert L.meu_slab_fft_create(32, 48, 64, 5, 0, P.PREC_F64, C.byref(h)) == badarg  # 5 divides neither
    assert L.meu_slab_fft_create(32, 48, 64, 2, 2, P.PREC_F64, C.byref(h)) == badarg  # rank outside [0, P)
    assert L.meu_slab_fft_create(32, 48, 64, 2, 0, 7, C.byref(h)) == badarg  # no such precision
    assert L.meu_slab_fft_create(32, 40, 64, 2, 0, P.PREC_F64, C.byref(h)) == unsupported  # Ny/P = 20 = 2^2 5


@pytest.mark.gpu
@pytest.mark.parametrize("with_group", [False, True])
def test_slabfft_driver_one_rank(with_group, tmp_path):
    import torch
    import torch.distributed as dist

    from meumapps_ss_b200.slab_fft import SlabFFT

    nx, ny, nz = SHAPE
    if with_group:
        dist.init_process_group("nccl", init_method=f"file://{tmp_path}/pg", rank=0, world_size=1)
    try:
        f = SlabFFT(nx, ny, nz, precision=P.PREC_F64)
        x = _full(P.PREC_F64, seed=9)
        real = torch.tensor(x, dtype=torch.float64, device="cuda")
        k = f.forward(real)
        ref = np.fft.rfftn(x, axes=(0, 1, 2)) / (nx * ny * nz)
        assert np.max(np.abs(k.cpu().numpy() - ref)) <= 1e-12 * np.max(np.abs(ref))
        back = f.inverse(k)
        assert np.max(np.abs(back.cpu().numpy() - x)) <= 1e-11 * np.max(np.abs(x))
        f.close()
    finally:
        if with_group:
            dist.destroy_process_group()
