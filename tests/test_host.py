"""Host-side set-up: Input.txt reader, parameter transforms, ran_2 (CPU)."""
import ctypes as C
import math

import numpy as np
import pytest

from meumapps_ss_b200 import _lib
from meumapps_ss_b200 import configs as CF
from meumapps_ss_b200 import params as P


def test_ran2_three_restatements_agree(oracle):
    for seed in (-1, -7, -11, -96, -123456, 0, 5):
        a, b, c = P.Ran2(seed), _lib.Ran2(seed), oracle.OracleRan2(seed)
        for _ in range(200):
            x, y, z = a(), b(), c()
            assert x == y == z
            assert 0.0 < x < 1.0


def test_ran2_constants():
    # am = 1./im1 is evaluated in REAL*4: float(2147483563) rounds to 2**31 - 128
    # and the quotient is rounded to REAL*4 before it widens to the REAL*8 parameter
    assert float(np.float32(2147483563)) == 2.0 ** 31 - 128
    assert P.Ran2.AM == float(np.float32(1.0) / np.float32(2.0 ** 31 - 128))
    assert P.Ran2.AM != 2.0 ** -31
    assert P.Ran2.RNMX == 1.0 - 1.2e-7


def test_langevin_agrees(oracle):
    b, c = _lib.Ran2(-9), oracle.OracleRan2(-9)
    vals = [b.langevin(0.3) for _ in range(2000)]
    ref = [c.langevin(0.3) for _ in range(2000)]
    assert vals == ref
    assert abs(np.std(vals) - 0.3) < 0.03


def test_langevin_fill_equals_serial_draws():
    # meu_langevin_fill (the chain on one thread, the logarithms on several) gives the
    # numbers and the final state of as many meu_langevin calls, fresh seed or not
    for seed, n, threads, pre in ((-5, 300000, 4, 0), (-12, 70001, 3, 17), (-3, 5, 8, 1), (-8, 0, 2, 2)):
        a, b = _lib.Ran2(seed), _lib.Ran2(seed)
        for _ in range(pre):
            a.langevin(0.5)
            b.langevin(0.5)
        ser = np.array([a.langevin(0.02) for _ in range(n)])
        got = b.langevin_fill(0.02, n, threads)
        assert np.array_equal(ser, got), (seed, n)
        assert bytes(a.s) == bytes(b.s)
        assert a() == b()


def test_oracle_initialiser_matches_library(oracle):
    # the CPU legs of the benchmark draw their inputs with the oracle's own ran_2
    for args in ((16, 16, 16, 3, -7, 0.2, 0.01, 0.001), (12, 8, 6, 1, -1, 0.15, 0.01, 0.001)):
        c1, e1 = _lib.init_uniform(*args)
        c2, e2 = oracle.init_uniform(*args)
        assert np.array_equal(c1, c2) and np.array_equal(e1, e2)


def test_init_uniform_matches_python():
    from helpers import py_uniform
    c, e = _lib.init_uniform(6, 5, 4, 3, -7, 0.2, 0.01, 0.001)
    c2, e2 = py_uniform(6, 5, 4, 3, -7, 0.2, 0.01, 0.001)
    assert np.array_equal(c, c2) and np.array_equal(e, e2)
    assert abs(c.mean() - 0.2) < 0.01 and np.abs(e).max() <= 0.001


def test_input_txt_and_setup():
    deck = P.parse_input_txt(CF.kks_input_txt(16, 3, 7))
    assert (deck.nx, deck.ny, deck.nz, deck.vartot, deck.numph, deck.numel_in) == (16, 16, 16, 3, 2, 2)
    p = P.kks_params(deck)
    mv = float(np.float32(1.055e-5))
    assert p.gparams[0][0] == pytest.approx(2.0e4 / mv)
    assert p.gparams[1][1] == pytest.approx(-600.0 / mv)
    assert p.gparams[1][2] == 0.55  # equilibrium composition is not scaled
    # 3 variants: axis permutations of TStr (ModInitials.f:171-186)
    tr = [[p.trans_ppt[v][i] for i in range(3)] for v in range(3)]
    assert tr == [[0.02, -0.005, -0.005], [-0.005, 0.02, -0.005], [-0.005, -0.005, 0.02]]
    # SEla = CEla^-1 and cubic completion
    cm, sm = p.matrix("cela", 0, 6), p.matrix("sela", 0, 6)
    assert np.allclose(cm @ sm, np.eye(6))
    assert cm[1, 1] == cm[0, 0] and cm[4, 4] == cm[3, 3] and cm[0, 2] == cm[0, 1]
    b_width = 5.0 * 1.0e-9
    assert p.wellph[1] == pytest.approx(6.0 * 0.3 / b_width)
    assert p.grad_coeff[0][0] == pytest.approx(b_width * 0.1 / 1e-18)
    assert p.cmobs[0] == pytest.approx(1e-16 / 1e-18)


def test_input_errors():
    txt = CF.kks_input_txt(16, 3, 7).replace("2 3 1\n", "2 2 1\n")
    with pytest.raises(P.SetupError) as e:
        P.parse_input_txt(txt)
    assert e.value.code == 1


def test_init_fields_single_nucleus():
    deck = P.parse_input_txt(CF.kks_input_txt(16, 1, 5, radius=3))
    cons, phi = P.init_fields(deck)
    assert phi.shape == (1, 16, 16, 16)
    assert phi[0, 7, 7, 7] == 1.0 and phi[0, 0, 0, 0] == 0.0
    # cppt: concentration Cimax inside the nucleus
    assert cons[0, 7, 7, 7] == 0.55 and cons[0, 0, 0, 0] == 0.15


def test_fortran_layout_roundtrip():
    a = np.arange(2 * 3 * 4 * 5, dtype=float).reshape(2, 3, 4, 5)
    f = P.to_fortran(a)
    assert f[0] == a[0, 0, 0, 0] and f[1] == a[1, 0, 0, 0] and f[2] == a[0, 0, 0, 1]
    assert np.array_equal(P.from_fortran(f, 2, 5, 4, 3), a)


@pytest.mark.parametrize("nvar,numel_in", [(1, 2), (3, 2), (3, 3)])
def test_params_from_gparams_matches_host_setup(nvar, numel_in):
    """The C fill of meu_params from the ModGparams arrays (Fortran layout) gives
    the same block, byte for byte, as the host restatement of the set-up."""
    deck = P.parse_input_txt(CF.kks_input_txt(16, nvar, 5, numel_in=numel_in))
    ref = P.kks_params(deck)
    V, E, NP = ref.nvar, ref.numel, ref.numph
    f = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F"))  # noqa: E731
    grad = np.zeros((3, 3, V), order="F")
    trans = np.zeros((6, V), order="F")
    for v in range(V):
        grad[:, :, v] = np.array(ref.grad_coeff[v][:]).reshape(3, 3, order="F")
        trans[:, v] = ref.trans_ppt[v][:]
    cela = np.zeros((6, 6, NP), order="F")
    sela = np.zeros((6, 6, NP), order="F")
    gpar = np.zeros((2 * E + 1, NP), order="F")
    for n in range(NP):
        cela[:, :, n] = ref.matrix("cela", n, 6)
        sela[:, :, n] = ref.matrix("sela", n, 6)
        gpar[:, n] = ref.gparams[n][:2 * E + 1]
    arrays = [f([ref.cmobs[e] for e in range(E)]), f(ref.e_mean[:]), f(grad), f(trans), f(cela), f(sela), f(gpar),
              f(ref.wellph[:NP])]
    nv = (C.c_int32 * NP)(*[ref.nvar_ph[n] for n in range(NP)])
    out = P.MeuParams()
    st = _lib.lib().meu_params_from_gparams(ref.nx, ref.ny, ref.nz, V, E, NP, nv, ref.step, ref.elastep0,
                                            ref.noise_step, ref.dt, ref.b_mob,
                                            *[_lib.dptr(a) for a in arrays], C.byref(out))
    assert st == 0
    assert bytes(out) == bytes(ref)
    assert _lib.lib().meu_params_from_gparams(16, 16, 16, 99, E, NP, nv, 1, 1, 0, 1.0, 1.0,
                                              *[_lib.dptr(a) for a in arrays], C.byref(out)) == 100
