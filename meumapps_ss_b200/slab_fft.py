"""Slab-decomposed 3-D real FFT of one grid over P GPUs, one process per GPU
(``meu_slab_fft_*`` in include/meu.h, ``csrc/slab_fft.cu``).

The reference splits its grid into P3DFFT pencils (Multi_MEUMAPPS.f:124-128,
:241-248) and calls f_trans / inv_trans (ModFunc.f:15-40) on them.  Here a grid
too large for one GPU is split into z slabs, and each transform makes one
all-to-all of P equal chunks (NCCL over NVLink, through torch.distributed).

Layout contract (the CUDA pack / unpack kernels implement it):

* rank r holds the real z-planes [r*NZL, (r+1)*NZL) as ``real[z][y][x]``
  (NZL = Nz/P) and, after ``forward``, the ky rows [r*NYL, (r+1)*NYL) of the
  scaled half spectrum as ``kslab[kz][ky][kx]`` (NYL = Ny/P, kx in [0, Nx/2]);
* the forward send buffer holds P chunks; chunk d = the rank's planes' (x R2C,
  y FFT) spectrum at d's ky rows, ``[z][ky][kx]``, times 1/P; chunk q received
  from rank q is the k-slab's z rows of rank q, so the receive buffer IS the
  k-slab before its z FFT;
* the inverse sends chunk q of the (z-inverted) k-slab to rank q and unpacks
  the chunk received from rank d into the planes' ky rows of d.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

from . import params as P
from ._lib import MeuError, lib


def slab_geometry(nx: int, ny: int, nz: int, nranks: int) -> dict:
    """Slab sizes of a (Nx, Ny, Nz) grid on nranks ranks."""
    if ny % nranks or nz % nranks:
        raise ValueError("Ny and Nz must be multiples of the rank count")
    return {"nzl": nz // nranks, "nyl": ny // nranks, "nxh": nx // 2 + 1, "P": nranks}


def exchange(send, recv, group=None) -> None:
    """The transform's all-to-all: chunk q of ``send`` to rank q, chunk q of
    ``recv`` from rank q (P equal chunks along the first dimension).  Complex
    tensors travel as their real view.  Without a process group (one rank) it is
    a copy."""
    import torch
    import torch.distributed as dist

    s = torch.view_as_real(send) if send.is_complex() else send
    r = torch.view_as_real(recv) if recv.is_complex() else recv
    if dist.is_available() and dist.is_initialized():
        dist.all_to_all_single(r, s, group=group)
    else:
        r.copy_(s)


class SlabFFT:
    """f_trans / inv_trans of a grid whose z-planes are split over the ranks of
    ``group`` (or one rank without torch.distributed).  Inputs and outputs are
    CUDA tensors of this rank; work runs on the current torch stream."""

    def __init__(self, nx: int, ny: int, nz: int, precision: int = P.PREC_F32, group=None,
                 device: Optional[str] = None):
        import torch
        import torch.distributed as dist

        if dist.is_available() and dist.is_initialized():
            nranks, rank = dist.get_world_size(group), dist.get_rank(group)
        else:
            nranks, rank = 1, 0
        self.group = group
        self.nx, self.ny, self.nz, self.precision = nx, ny, nz, precision
        self.geo = slab_geometry(nx, ny, nz, nranks)
        self.rank, self.nranks = rank, nranks
        h = C.c_void_p()
        st = lib().meu_slab_fft_create(nx, ny, nz, nranks, rank, precision, C.byref(h))
        if st:
            raise MeuError(st, lib().meu_last_error(None).decode())
        self.h = h
        self.rdtype = torch.float64 if precision == P.PREC_F64 else torch.float32
        self.cdtype = torch.complex128 if precision == P.PREC_F64 else torch.complex64
        self.device = torch.device(device) if device else torch.device("cuda", torch.cuda.current_device())
        g = self.geo
        self.kslab_shape = (nz, g["nyl"], g["nxh"])
        self.real_shape = (g["nzl"], ny, nx)
        self._buf = torch.empty(self.kslab_shape, dtype=self.cdtype, device=self.device)

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().meu_slab_fft_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int) -> None:
        if st:
            raise MeuError(st, lib().meu_slab_fft_last_error(self.h).decode())

    def _stream(self):
        import torch

        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def forward(self, real):
        """Real slab (NZL, Ny, Nx) -> this rank's k-slab (Nz, NYL, Nx/2+1), scaled by 1/(Nx Ny Nz)."""
        import torch

        if tuple(real.shape) != self.real_shape or real.dtype != self.rdtype or not real.is_contiguous():
            raise ValueError(f"real slab must be a contiguous {self.rdtype} tensor of shape {self.real_shape}")
        st = self._stream()
        self._check(lib().meu_slab_fft_forward_planes(self.h, C.c_void_p(real.data_ptr()),
                                                      C.c_void_p(self._buf.data_ptr()), st))
        kslab = torch.empty(self.kslab_shape, dtype=self.cdtype, device=self.device)
        exchange(self._buf, kslab, self.group)
        self._check(lib().meu_slab_fft_forward_columns(self.h, C.c_void_p(kslab.data_ptr()), st))
        return kslab

    def inverse(self, kslab):
        """This rank's k-slab -> real slab, unscaled (inv_trans).  kslab is used as
        scratch and holds garbage afterwards."""
        import torch

        if tuple(kslab.shape) != self.kslab_shape or kslab.dtype != self.cdtype or not kslab.is_contiguous():
            raise ValueError(f"k-slab must be a contiguous {self.cdtype} tensor of shape {self.kslab_shape}")
        st = self._stream()
        self._check(lib().meu_slab_fft_inverse_columns(self.h, C.c_void_p(kslab.data_ptr()), st))
        exchange(kslab, self._buf, self.group)
        real = torch.empty(self.real_shape, dtype=self.rdtype, device=self.device)
        self._check(lib().meu_slab_fft_inverse_planes(self.h, C.c_void_p(self._buf.data_ptr()),
                                                      C.c_void_p(real.data_ptr()), st))
        return real
