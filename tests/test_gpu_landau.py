"""Landau decks: GPU plain FP64 against the CPU FP64 oracle (<= 1e-10 max-abs),
and the FP32 bulk path against the GPU FP64 path (stated relative L2 bounds)."""
import numpy as np
import pytest

from helpers import active_landau, py_uniform
from meumapps_ss_b200 import configs as CF
from meumapps_ss_b200 import params as P
from meumapps_ss_b200.sim import Simulation

TOL = 1e-10


def _pair(oracle, p, c, e, steps, chunks=1):
    o = oracle.OracleSim(p)
    o.set_fields(c, e)
    g = Simulation(p)
    g.set_fields(c, e)
    do, dg = [], []
    for _ in range(chunks):
        do.append(o.run(steps // chunks))
        dg.append(g.run(steps // chunks))
    cat = lambda ds, k: np.concatenate([d[k] for d in ds])
    return o, g, do, dg, cat


@pytest.mark.gpu
@pytest.mark.parametrize("nvar,elastic,coupling", [(1, P.ELAST_HOMOG, P.EIG_ETA2), (3, P.ELAST_HOMOG, P.EIG_ETA2),
                                                   (2, P.ELAST_NONE, P.EIG_ETA2), (1, P.ELAST_HOMOG, P.EIG_H)])
def test_landau_active_parity(oracle, nvar, elastic, coupling):
    p, c, e = active_landau(n=16, nvar=nvar, elastic=elastic, coupling=coupling)
    o, g, do, dg, cat = _pair(oracle, p, c, e, 100, chunks=2)
    co, eo, _, _ = o.get_fields()
    cg, eg, _, _ = g.get_fields()
    assert np.max(np.abs(cg - co)) <= TOL
    assert np.max(np.abs(eg - eo)) <= TOL
    assert np.max(np.abs(eo - e)) > 1e-2  # the deck really evolves
    for k in ("fint", "fch", "elen", "etot", "cmin", "cmax", "phimax", "solid_now"):
        a, b = cat(do, k), cat(dg, k)
        assert np.max(np.abs(a - b) / np.maximum(np.abs(a), 1e-30)) < 1e-9, k
    assert np.max(np.abs(cat(dg, "cavg")[:, 0] - c.mean())) < 1e-14


@pytest.mark.gpu
def test_landau_hetero_parity(oracle):
    p, c, e = active_landau(n=16, nvar=2, elastic=P.ELAST_HETERO, coupling=P.EIG_H, ppt_scale=1.5, el_tol=1e-8)
    o, g, do, dg, cat = _pair(oracle, p, c, e, 40, chunks=2)
    assert np.array_equal(cat(do, "el_iters"), cat(dg, "el_iters"))
    co, eo, elo, _ = o.get_fields()
    cg, eg, elg, _ = g.get_fields()
    assert np.max(np.abs(cg - co)) <= TOL and np.max(np.abs(eg - eo)) <= TOL
    assert np.max(np.abs(elg - elo)) <= 1e-9 * np.max(np.abs(elo))


@pytest.mark.gpu
@pytest.mark.parametrize("ortho,pv,ct", [(True, 0, 1), (False, 2, 2)])
def test_landau_hetero_kernels_parity(oracle, ortho, pv, ct):
    """Proportional moduli through the matrix-free kernels on a 64^3 grid (the
    compile-time transforms), with the normal / shear blocks decoupled (cubic) or
    coupled (an off-block term added to the stiffness), under both radix plans."""
    p, c, e = active_landau(n=64, nvar=2, elastic=P.ELAST_HETERO, coupling=P.EIG_H, ppt_scale=1.5, el_tol=1e-8)
    if not ortho:
        cm = p.matrix("cela", 0, 6)
        cm[0, 3] = cm[3, 0] = 7.0
        cm[1, 5] = cm[5, 1] = -4.0
        for ph, scale in ((0, 1.0), (1, 1.0 / 1.5)):
            p.set_matrix("cela", ph, cm / scale)
            p.set_matrix("sela", ph, np.linalg.inv(cm / scale))
    o = oracle.OracleSim(p)
    o.set_fields(c, e)
    g = Simulation(p)
    g.set_schedule(pv, 0, ct)
    g.set_fields(c, e)
    do, dg = o.run(6), g.run(6)
    assert np.array_equal(do["el_iters"], dg["el_iters"])
    co, eo, elo, _ = o.get_fields()
    cg, eg, elg, _ = g.get_fields()
    assert np.max(np.abs(cg - co)) <= TOL and np.max(np.abs(eg - eo)) <= TOL
    assert np.max(np.abs(elg - elo)) <= 1e-9 * np.max(np.abs(elo))


@pytest.mark.gpu
@pytest.mark.parametrize("ny,nz", [(12, 9), (32, 48)])
def test_landau_hetero_fused_rows_noncubic_parity(oracle, ny, nz):
    """Fused elastic rows on non-cubic grids against the oracle in FP64: 12 x 9 = 108
    rows leave a partial last block of rows; nz = 48 runs the run-time z plan."""
    p, _, _ = active_landau(n=64, nvar=2, elastic=P.ELAST_HETERO, coupling=P.EIG_H, ppt_scale=1.5, el_tol=1e-8)
    p.ny, p.nz = ny, nz
    c, e = py_uniform(64, ny, nz, 2, -5, 0.8, 0.05, 0.5)
    o = oracle.OracleSim(p)
    o.set_fields(c, e)
    do = o.run(4)
    with Simulation(p) as g:
        g.set_fields(c, e)
        g.timing(True)
        dg = g.run(4)
        assert "el_rows" in g.timing_report()
        cg, eg, elg, _ = g.get_fields()
    co, eo, elo, _ = o.get_fields()
    assert np.array_equal(do["el_iters"], dg["el_iters"])
    assert np.max(np.abs(cg - co)) <= TOL and np.max(np.abs(eg - eo)) <= TOL
    assert np.max(np.abs(elg - elo)) <= 1e-9 * np.max(np.abs(elo))


@pytest.mark.gpu
def test_landau_hetero_fused_rows_many_variants_parity(oracle):
    """Six variants: more order parameters than the fused rows prefetch into shared
    memory, so the polarisation reads them from global memory; FP64 against the oracle."""
    p, c, e = active_landau(n=64, nvar=6, elastic=P.ELAST_HETERO, coupling=P.EIG_H, ppt_scale=1.5, el_tol=1e-8)
    p.ny, p.nz = 16, 16
    c, e = py_uniform(64, 16, 16, 6, -3, 0.8, 0.05, 0.5)
    o = oracle.OracleSim(p)
    o.set_fields(c, e)
    do = o.run(3)
    with Simulation(p) as g:
        g.set_fields(c, e)
        g.timing(True)
        dg = g.run(3)
        assert "el_rows" in g.timing_report()
        cg, eg, _, _ = g.get_fields()
    co, eo, _, _ = o.get_fields()
    assert np.array_equal(do["el_iters"], dg["el_iters"])
    assert np.max(np.abs(cg - co)) <= TOL and np.max(np.abs(eg - eo)) <= TOL


@pytest.mark.gpu
def test_landau_hetero_fp32_fused_rows():
    """FP32 heterogeneous step on 64^3, where each fixed-point iteration runs its x
    transforms and the polarisation as one kernel, against the FP64 step."""
    p64, c, e = active_landau(n=64, nvar=2, elastic=P.ELAST_HETERO, coupling=P.EIG_H, ppt_scale=1.5, el_tol=1e-8)
    p32 = p64.copy()
    p32.precision = P.PREC_F32
    out = {}
    for name, p in (("f64", p64), ("f32", p32)):
        with Simulation(p) as g:
            g.set_fields(c, e)
            g.timing(True)
            g.run(10)
            assert "el_rows" in g.timing_report()
            out[name] = g.get_fields()
    rc = np.linalg.norm(out["f32"][0] - out["f64"][0]) / np.linalg.norm(out["f64"][0])
    re = np.linalg.norm(out["f32"][1] - out["f64"][1]) / np.linalg.norm(out["f64"][1])
    rl = np.linalg.norm(out["f32"][2] - out["f64"][2]) / np.linalg.norm(out["f64"][2])
    assert rc <= 1e-5 and re <= 1e-5 and rl <= 1e-4, (rc, re, rl)


@pytest.mark.gpu
def test_landau_hetero_fp32_odd_cell_count():
    """FP32 heterogeneous step on an 18 x 9 x 9 grid: 1458 cells is no multiple of four
    floats, so the elastic kernels copy their tiles element by element; checked
    against the FP64 step (16-byte copies) of the same deck."""
    p64, _, _ = active_landau(n=18, nvar=2, elastic=P.ELAST_HETERO, coupling=P.EIG_H, ppt_scale=1.5, el_tol=1e-8)
    p64.ny, p64.nz = 9, 9
    c, e = py_uniform(18, 9, 9, 2, -3, 0.8, 0.05, 0.5)
    p32 = p64.copy()
    p32.precision = P.PREC_F32
    out = {}
    for name, p in (("f64", p64), ("f32", p32)):
        with Simulation(p) as g:
            g.set_fields(c, e)
            g.run(20)
            out[name] = g.get_fields()
    rc = np.linalg.norm(out["f32"][0] - out["f64"][0]) / np.linalg.norm(out["f64"][0])
    re = np.linalg.norm(out["f32"][1] - out["f64"][1]) / np.linalg.norm(out["f64"][1])
    rl = np.linalg.norm(out["f32"][2] - out["f64"][2]) / np.linalg.norm(out["f64"][2])
    assert rc <= 1e-5 and re <= 1e-5 and rl <= 1e-4, (rc, re, rl)


@pytest.mark.gpu
@pytest.mark.parametrize("k", [0, 1, 2])
def test_landau_configs_small_parity(oracle, k):
    w = CF.landau_config(k, n=16, precision=P.PREC_F64)
    c, e = py_uniform(16, 16, 16, w.params.nvar, w.seed, w.c0, w.c_amp, w.eta_amp)
    o, g, do, dg, cat = _pair(oracle, w.params, c, e, 30)
    co, eo, _, _ = o.get_fields()
    cg, eg, _, _ = g.get_fields()
    assert np.max(np.abs(cg - co)) <= TOL and np.max(np.abs(eg - eo)) <= TOL


@pytest.mark.gpu
@pytest.mark.parametrize("nvar", [1, 3])
def test_fp32_bulk_vs_fp64(nvar):
    p64, c, e = active_landau(n=32, nvar=nvar, elastic=P.ELAST_HOMOG)
    p32 = p64.copy()
    p32.precision = P.PREC_F32
    out = {}
    for name, p in (("f64", p64), ("f32", p32)):
        with Simulation(p) as g:
            g.set_fields(c, e)
            d = g.run(200)
            out[name] = (g.get_fields(), d)
    (c64, e64, _, _), d64 = out["f64"]
    (c32, e32, _, _), d32 = out["f32"]
    rc = np.linalg.norm(c32 - c64) / np.linalg.norm(c64)
    re = np.linalg.norm(e32 - e64) / np.linalg.norm(e64)
    assert rc < 1e-5 and re < 1e-4, (rc, re)
    # FP64 k = 0 mode and reductions keep the mean concentration exact
    assert np.max(np.abs(d32["cavg"][:, 0] - c.mean())) < 1e-7


@pytest.mark.gpu
def test_single_mode_decay_exact():
    """Linear operator known answer: with a zero local free energy one Fourier
    mode of eta decays by exactly 1/(1 + dt L kappa k^2) per step and one mode
    of c by 1/(1 + dt M kappa_c k^4)."""
    n = 32
    p = CF.landau_params(n, 1, [[0, 0, 0]], elastic=P.ELAST_NONE, A=0.0, B=0.0, Cq=0.0, D=0.0, dt=0.05,
                         kappa_eta=1.3, kappa_c=0.7, M=0.9, L=1.1)
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    k = 2 * np.pi * np.sqrt(2.0 ** 2 + 3.0 ** 2) / n
    mode = np.cos(2 * np.pi * (2 * x + 3 * y) / n)
    c = 0.3 + 0.01 * mode
    e = 0.02 * mode
    with Simulation(p) as g:
        g.set_fields(c[None], e[None])
        g.run(10)
        cg, eg, _, _ = g.get_fields()
    fe = (1.0 / (1.0 + 0.05 * 1.1 * 1.3 * k * k)) ** 10
    fc = (1.0 / (1.0 + 0.05 * 0.9 * 0.7 * k ** 4)) ** 10
    assert np.max(np.abs(eg[0] - 0.02 * fe * mode)) < 1e-14
    assert np.max(np.abs(cg[0] - (0.3 + 0.01 * fc * mode))) < 1e-14
