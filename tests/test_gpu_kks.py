"""KKS model: the GPU plain-FP64 step against the CPU FP64 oracle, which
restates Multi_MEUMAPPS.f:548-1106 and ModElastic.f.  Gate: <= 1e-10 max-abs
on the fields over the first 100 steps."""
import numpy as np
import pytest

from helpers import kks_case
from meumapps_ss_b200 import params as P
from meumapps_ss_b200.sim import Simulation

TOL = 1e-10


def _run_both(oracle, p, cons, phi, steps, chunks=1, ustate=None):
    o = oracle.OracleSim(p)
    o.set_fields(cons, phi, ustate)
    g = Simulation(p)
    g.set_fields(cons, phi, ustate)
    per = steps // chunks
    do, dg = [], []
    for _ in range(chunks):
        do.append(o.run(per))
        dg.append(g.run(per))
    return o, g, do, dg


def _cat(ds, k):
    return np.concatenate([d[k] for d in ds])


@pytest.mark.gpu
@pytest.mark.parametrize("nvar,n", [(1, 16), (3, 16), (1, 24)])
def test_kks_fields_parity_100_steps(oracle, nvar, n):
    _, p, cons, phi = kks_case(n=n, nvar=nvar, steps=100)
    o, g, do, dg = _run_both(oracle, p, cons, phi, 100, chunks=4)
    co, fo, eo, uo = o.get_fields()
    cg, fg, eg, ug = g.get_fields(ustate=True)
    assert np.max(np.abs(cg - co)) <= TOL
    assert np.max(np.abs(fg - fo)) <= TOL
    assert np.max(np.abs(ug - uo)) <= TOL * max(1.0, np.max(np.abs(uo)))
    assert np.max(np.abs(eg - eo)) <= 1e-9 * np.max(np.abs(eo))
    assert np.array_equal(_cat(do, "el_iters"), _cat(dg, "el_iters"))
    for k in ("fint", "fw", "fch", "elen", "etot"):
        a, b = _cat(do, k), _cat(dg, k)
        assert np.max(np.abs(a - b) / np.maximum(np.abs(a), 1e-300)) < 1e-9, k
    for k in ("cmin", "cmax", "phimax", "solid_now", "glob_min", "glob_max", "phi_max", "solid"):
        assert np.max(np.abs(_cat(do, k) - _cat(dg, k))) <= TOL, k
    assert np.max(np.abs(_cat(do, "cavg") - _cat(dg, "cavg"))) <= 1e-13
    assert g.step == o.step == p.step + 100


@pytest.mark.gpu
def test_kks_two_solutes_parity(oracle):
    _, p, cons, phi = kks_case(n=16, nvar=1, steps=30, numel_in=3)
    assert p.numel == 2
    o, g, _, _ = _run_both(oracle, p, cons, phi, 30)
    co, fo, _, _ = o.get_fields()
    cg, fg, _, _ = g.get_fields()
    assert np.max(np.abs(cg - co)) <= TOL and np.max(np.abs(fg - fo)) <= TOL


@pytest.mark.gpu
def test_kks_noise_and_restart_state(oracle):
    _, p, cons, phi = kks_case(n=16, nvar=3, steps=20)
    p.noise_step = p.step + 4
    from meumapps_ss_b200._lib import Ran2
    rng = Ran2(-17)
    o = oracle.OracleSim(p)
    o.set_fields(cons, phi)
    g = Simulation(p)
    g.set_fields(cons, phi)
    for s in range(8):
        incr = np.array([rng.langevin(1e-3) for _ in range(phi.size)]).reshape(phi.shape[1:] + (3,))
        incr = np.moveaxis(incr, -1, 0)
        o.add_noise(incr)
        g.add_noise(incr)
        o.run(1)
        g.run(1)
    _, fo, _, uo = o.get_fields()
    _, fg, _, ug = g.get_fields(ustate=True)
    assert np.max(np.abs(fg - fo)) <= TOL
    # restart through the data_save state (u, grad u): both continue identically
    c1, f1, _, _ = o.get_fields()
    p2 = p.copy()
    p2.step = o.step
    o2 = oracle.OracleSim(p2)
    o2.set_fields(c1, f1, uo)
    g2 = Simulation(p2)
    g2.set_fields(c1, f1, ug)
    o2.run(5)
    g2.run(5)
    assert np.max(np.abs(g2.get_fields()[1] - o2.get_fields()[1])) <= TOL


@pytest.mark.gpu
def test_kks_mass_conservation_and_clip():
    _, p, cons, phi = kks_case(n=16, nvar=3, steps=50)
    with Simulation(p) as g:
        g.set_fields(cons, phi)
        d = g.run(50)
        c, f, _, _ = g.get_fields()
    assert np.max(np.abs(d["cavg"][:, 0] - cons.mean())) < 1e-13
    assert f.min() >= 0.0 and f.max() <= 1.0


@pytest.mark.gpu
def test_kks_rejects_bad_sizes_and_precision():
    from meumapps_ss_b200._lib import MeuError
    _, p, _, _ = kks_case(n=16)
    q = p.copy()
    q.nx = 10
    with pytest.raises(MeuError) as e:
        Simulation(q)
    assert e.value.code == 103
    q = p.copy()
    q.precision = 7
    with pytest.raises(MeuError):
        Simulation(q)


@pytest.mark.gpu
def test_kks_equal_moduli_parity(oracle):
    # matrix and precipitate share one stiffness: the per-voxel compliance mix
    # reduces to a scalar multiple of the matrix's (the scalar-mix path)
    _, p, cons, phi = kks_case(n=16, nvar=3, steps=40, hetero=False)
    o, g, do, dg = _run_both(oracle, p, cons, phi, 40)
    co, fo, eo, _ = o.get_fields()
    cg, fg, eg, _ = g.get_fields()
    assert np.max(np.abs(cg - co)) <= TOL and np.max(np.abs(fg - fo)) <= TOL
    assert np.max(np.abs(eg - eo)) <= 1e-9 * np.max(np.abs(eo))
    assert np.array_equal(_cat(do, "el_iters"), _cat(dg, "el_iters"))


def _kks12(n, precision=P.PREC_F64, steps=30):
    from meumapps_ss_b200 import configs as CF
    deck = P.parse_input_txt(CF.kks_input_txt(n, 12, steps, radius=4))
    p = P.kks_params(deck, precision=precision, sym_var=CF.tetrahedral_rotations())
    cons, phi = P.init_fields(deck)
    return p, cons, phi


@pytest.mark.gpu
def test_kks_12_variants_parity(oracle):
    # 12 orientation variants (sym_var rotations), heterogeneous moduli, plain FP64
    p, cons, phi = _kks12(16)
    assert p.nvar == 12
    o, g, do, dg = _run_both(oracle, p, cons, phi, 30)
    co, fo, _, _ = o.get_fields()
    cg, fg, _, _ = g.get_fields()
    assert np.max(np.abs(cg - co)) <= TOL and np.max(np.abs(fg - fo)) <= TOL
    assert np.array_equal(_cat(do, "el_iters"), _cat(dg, "el_iters"))


@pytest.mark.gpu
def test_kks_12_variants_fp32_against_fp64():
    # the reference's production shape (12 variants) with FP32 fields: relative L2
    # of the concentration and of the order parameters against the plain FP64 path
    out = {}
    for prec in (P.PREC_F64, P.PREC_F32):
        p, cons, phi = _kks12(32, prec, 200)
        g = Simulation(p)
        g.set_fields(cons, phi)
        g.run(200, diag=False)
        out[prec] = g.get_fields()
    c64, f64, _, _ = out[P.PREC_F64]
    c32, f32, _, _ = out[P.PREC_F32]
    rc = np.linalg.norm(c32 - c64) / np.linalg.norm(c64)
    rf = np.linalg.norm(f32 - f64) / np.linalg.norm(f64)
    print("kks12 fp32 rel", rc, rf)
    assert rc <= 1e-5 and rf <= 1e-4, (rc, rf)


@pytest.mark.gpu
def test_run_noise_matches_serial_draws(oracle):
    """meu_run_noise (host thread drawing the next step's increments while a step runs)
    against serial langevin draws passed to meu_add_noise before each single step: the
    same fields bit for bit, the same final ran_2 state, and the oracle within 1e-10."""
    import ctypes as C
    from meumapps_ss_b200._lib import Ran2, Ran2State, dptr, lib
    _, p, cons, phi = kks_case(n=16, nvar=3, steps=20)
    p.noise_step = p.step + 4  # 5 noisy steps, then 3 without
    sd, seed, steps = 2e-3, -23, 8
    r1 = Ran2(seed)
    o = oracle.OracleSim(p)
    o.set_fields(cons, phi)
    with Simulation(p) as g1, Simulation(p) as g2:
        g1.set_fields(cons, phi)
        g2.set_fields(cons, phi)
        for s in range(steps):
            if g1.step <= p.noise_step:
                incr = np.array([r1.langevin(sd) for _ in range(phi.size)])  # Fortran order
                assert lib().meu_add_noise(g1.h, dptr(incr)) == 0
                o.add_noise(np.moveaxis(incr.reshape(phi.shape[1:] + (phi.shape[0],)), -1, 0))
            g1.run(1)
            o.run(1)
        st = Ran2State()
        lib().meu_ran2_init(C.byref(st), seed)
        g2.run_noise(steps, st, sd)
        c1, f1, _, _ = g1.get_fields()
        c2, f2, _, _ = g2.get_fields()
        assert np.array_equal(c1, c2) and np.array_equal(f1, f2)
        assert bytes(st) == bytes(r1.s)
        co, fo, _, _ = o.get_fields()
        assert np.max(np.abs(f2 - fo)) <= TOL and np.max(np.abs(c2 - co)) <= TOL
