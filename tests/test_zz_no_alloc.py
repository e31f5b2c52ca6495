"""The allocation-free transform entry point (meu_fft_roundtrip_noalloc).

Callers that cannot call cudaMalloc -- a driver whose device memory belongs to
its OpenACC / managed-memory runtime, or a framework whose allocator already
holds the GPU -- pass their own device arrays; the library works in a fixed
static device array instead of allocating.  These tests allocate the caller's
arrays with torch (the test is the caller) and check the entry point against
the allocating meu_fft_roundtrip on two calls in a row.  The file sorts last so
that a run stopping at the first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest

from meumapps_ss_b200 import _lib
from meumapps_ss_b200 import params as P

MAX_POINTS = 262144


def _noalloc(x, prec):
    import torch
    nz, ny, nx = x.shape
    d_in = torch.from_numpy(np.ascontiguousarray(x)).to("cuda")
    d_spec = torch.empty(2 * nz * ny * (nx // 2 + 1), dtype=torch.float64, device="cuda")
    d_back = torch.empty_like(d_in)
    st = _lib.lib().meu_fft_roundtrip_noalloc(nx, ny, nz, prec, C.c_void_p(d_in.data_ptr()),
                                             C.c_void_p(d_spec.data_ptr()), C.c_void_p(d_back.data_ptr()))
    assert st == 0, _lib.lib().meu_last_error(None)
    spec = d_spec.cpu().numpy().view(np.complex128).reshape(nz, ny, nx // 2 + 1)
    return spec, d_back.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [(P.PREC_F64, 1e-13), (P.PREC_F32, 1e-6)])
def test_noalloc_matches_allocating_entry_point(prec, tol):
    rng = np.random.default_rng(11)
    # two calls in a row on different grids: the shared static array keeps the
    # first call's contents, which must not leak into the second
    for shape in [(32, 32, 32), (16, 24, 48), (64, 64, 64)]:
        x = rng.standard_normal(shape)
        ref_spec, ref_back = _lib.fft_roundtrip(x, prec)
        spec, back = _noalloc(x, prec)
        assert np.linalg.norm(spec - ref_spec) <= tol * np.linalg.norm(ref_spec)
        assert np.linalg.norm(back - ref_back) <= tol * np.linalg.norm(ref_back)
        assert np.linalg.norm(back - x) <= 10 * tol * np.linalg.norm(x)


@pytest.mark.gpu
def test_noalloc_rejects_oversize_grid():
    import torch
    d = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = C.c_void_p(d.data_ptr())
    st = _lib.lib().meu_fft_roundtrip_noalloc(128, 64, 64, P.PREC_F64, p, p, p)
    assert st == 103
    assert b"exceed the maximum" in _lib.lib().meu_last_error(None)
    assert 128 * 64 * 64 > MAX_POINTS
