"""GPU transforms (through meu_fft_roundtrip) against numpy."""
import numpy as np
import pytest

from meumapps_ss_b200 import _lib
from meumapps_ss_b200 import params as P

# (nz, ny, nx).  Power-of-two lengths 32..512 (x: nx/2) take the compile-time
# kernels, the rest the run-time plan; the last three put lengths 512/256 on every
# axis and leave a partial column tile (ny = 512 with nx/2+1 = 9 columns).
SHAPES = [(8, 8, 8), (16, 16, 16), (12, 24, 6), (48, 48, 48), (32, 96, 64), (64, 64, 128), (128, 128, 128),
          (4, 6, 8), (9, 3, 12), (96, 96, 96), (16, 32, 1024), (512, 16, 36), (32, 512, 16), (256, 64, 512)]


@pytest.mark.gpu
@pytest.mark.parametrize("shape", SHAPES)
def test_fft_fp64(shape):
    rng = np.random.default_rng(5)
    x = rng.standard_normal(shape)
    spec, back = _lib.fft_roundtrip(x, P.PREC_F64)
    ref = np.fft.rfftn(x) / x.size
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(spec - ref)) <= 1e-14 * scale * np.log2(x.size)
    assert np.max(np.abs(back - x)) <= 1e-13 * np.max(np.abs(x))


@pytest.mark.gpu
@pytest.mark.parametrize("shape", SHAPES)
def test_fft_fp32(shape):
    rng = np.random.default_rng(6)
    x = rng.standard_normal(shape)
    spec, back = _lib.fft_roundtrip(x, P.PREC_F32)
    ref = np.fft.rfftn(x) / x.size
    rel = np.linalg.norm(spec - ref) / np.linalg.norm(ref)
    assert rel < 3e-7
    assert np.linalg.norm(back - x) / np.linalg.norm(x) < 5e-7


@pytest.mark.gpu
def test_fft_single_mode_exact():
    n = 32
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    f = np.cos(2 * np.pi * (3 * x + 5 * y - 2 * z) / n)
    spec, _ = _lib.fft_roundtrip(f, P.PREC_F64)
    mag = np.abs(spec)
    assert mag.max() == pytest.approx(0.5, abs=1e-14)
    assert np.sort(mag.ravel())[-2] == pytest.approx(0.0, abs=1e-14) or np.sum(mag > 1e-12) <= 2
