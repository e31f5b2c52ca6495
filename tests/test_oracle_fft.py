"""The oracle's f_trans / inv_trans and invert against numpy (CPU)."""
import numpy as np
import pytest


@pytest.mark.parametrize("shape", [(8, 8, 8), (6, 12, 16), (16, 24, 32), (48, 48, 48), (3, 9, 4)])
def test_rfft3_matches_numpy(oracle, shape):
    rng = np.random.default_rng(1)
    x = rng.standard_normal(shape)
    k = oracle.rfft3(x)
    ref = np.fft.rfftn(x) / x.size
    assert np.max(np.abs(k - ref)) < 1e-14 * max(1.0, np.max(np.abs(ref))) * 10


@pytest.mark.parametrize("shape", [(8, 8, 8), (6, 12, 16), (32, 32, 32), (96, 12, 48)])
def test_irfft3_roundtrip_and_c2r_semantics(oracle, shape):
    rng = np.random.default_rng(2)
    x = rng.standard_normal(shape)
    k = oracle.rfft3(x)
    back = oracle.irfft3(k, shape[2])
    assert np.max(np.abs(back - x)) < 1e-12
    # Im of the kx = 0 and kx = Nx/2 planes' self-conjugate points is discarded like FFTW c2r
    k2 = k.copy()
    k2[0, 0, 0] += 0.3j
    k2[0, 0, -1] += 0.7j
    assert np.max(np.abs(oracle.irfft3(k2, shape[2]) - back)) < 1e-12


def test_invert_and_condition_flag(oracle):
    rng = np.random.default_rng(3)
    for n in (2, 3, 6, 12):
        a = rng.standard_normal((n, n)) + n * np.eye(n)
        st, inv = oracle.invert(a)
        assert st == 0
        assert np.allclose(inv @ a, np.eye(n), atol=1e-12)
    st, _ = oracle.invert(np.ones((3, 3)))
    assert st != 0
