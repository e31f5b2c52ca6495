"""Fused Landau step (cubic N in {32,48,64,96,128}, 1-4 variants, eta^2
coupling): plain FP64 against the CPU FP64 oracle (<= 1e-10 max-abs, energies
to 1e-9 relative), and proof that the fused kernels are the ones that ran."""
import numpy as np
import pytest

from helpers import active_landau
from meumapps_ss_b200 import params as P
from meumapps_ss_b200.sim import Simulation

TOL = 1e-10


def _parity(oracle, p, c, e, steps, chunks=2):
    o = oracle.OracleSim(p)
    o.set_fields(c, e)
    g = Simulation(p)
    g.set_fields(c, e)
    g.timing(True)
    do, dg = [], []
    for _ in range(chunks):
        do.append(o.run(steps // chunks))
        dg.append(g.run(steps // chunks))
    names = set(g.timing_report())
    g.timing(False)
    co, eo, _, _ = o.get_fields()
    cg, eg, _, _ = g.get_fields()
    cat = lambda ds, k: np.concatenate([d[k] for d in ds])
    return co, eo, cg, eg, do, dg, cat, names


@pytest.mark.gpu
@pytest.mark.parametrize("nvar,elastic", [(1, P.ELAST_HOMOG), (2, P.ELAST_HOMOG), (3, P.ELAST_HOMOG),
                                          (4, P.ELAST_HOMOG), (3, P.ELAST_NONE)])
def test_fused_parity_32(oracle, nvar, elastic):
    p, c, e = active_landau(n=32, nvar=nvar, elastic=elastic)
    co, eo, cg, eg, do, dg, cat, names = _parity(oracle, p, c, e, 40)
    assert "lf_z_green_ch" in names and "lf_plane_fwd" in names
    assert np.max(np.abs(cg - co)) <= TOL
    assert np.max(np.abs(eg - eo)) <= TOL
    for k in ("fint", "fch", "elen", "etot", "cmin", "cmax", "phimax", "solid_now", "glob_min", "phi_max", "solid"):
        a, b = cat(do, k), cat(dg, k)
        assert np.max(np.abs(a - b) / np.maximum(np.abs(a), 1e-30)) < 1e-9, k
    assert np.max(np.abs(cat(dg, "cavg")[:, 0] - c.mean())) < 1e-14


@pytest.mark.gpu
@pytest.mark.parametrize("n,nvar", [(48, 1), (64, 2)])
def test_fused_parity_other_sizes(oracle, n, nvar):
    p, c, e = active_landau(n=n, nvar=nvar, elastic=P.ELAST_HOMOG)
    co, eo, cg, eg, do, dg, cat, names = _parity(oracle, p, c, e, 10, chunks=1)
    assert "lf_z_tdgl" in names
    assert np.max(np.abs(cg - co)) <= TOL and np.max(np.abs(eg - eo)) <= TOL


@pytest.mark.gpu
def test_fused_fp32_vs_fp64_128():
    """Config-1 shape (128^3, 3 variants) on the active deck: FP32 bulk against FP64."""
    p64, c, e = active_landau(n=128, nvar=3, elastic=P.ELAST_HOMOG, dt=0.005)
    p32 = p64.copy()
    p32.precision = P.PREC_F32
    res = {}
    for name, p in (("f64", p64), ("f32", p32)):
        with Simulation(p) as g:
            g.set_fields(c, e)
            d = g.run(200)
            res[name] = (g.get_fields(), d)
    (c64, e64, _, _), d64 = res["f64"]
    (c32, e32, _, _), d32 = res["f32"]
    rc = np.linalg.norm(c32 - c64) / np.linalg.norm(c64)
    re = np.linalg.norm(e32 - e64) / np.linalg.norm(e64)
    assert rc < 1e-5 and re < 1e-5, (rc, re)
    assert np.max(np.abs(d32["etot"] - d64["etot"]) / np.abs(d64["etot"])) < 1e-5


@pytest.mark.gpu
def test_config1_fp32_error_after_1000_steps():
    """Accuracy gate of the mixed-precision step: Landau deck 1 (128^3, 3
    variants, seed -7) after 1000 steps, FP32 bulk against the GPU's plain FP64
    path: relative L2 error <= 1e-5 in c and in eta."""
    from meumapps_ss_b200 import _lib
    from meumapps_ss_b200 import configs as CF
    w = CF.landau_config(1, precision=P.PREC_F64)
    c, e = _lib.init_uniform(128, 128, 128, 3, w.seed, w.c0, w.c_amp, w.eta_amp)
    out = {}
    for prec in (P.PREC_F64, P.PREC_F32):
        p = w.params.copy()
        p.precision = prec
        with Simulation(p) as g:
            g.set_fields(c, e)
            g.run(1000, diag=False)
            out[prec] = g.get_fields()
    c64, e64, _, _ = out[P.PREC_F64]
    c32, e32, _, _ = out[P.PREC_F32]
    rc = np.linalg.norm(c32 - c64) / np.linalg.norm(c64)
    re = np.linalg.norm(e32 - e64) / np.linalg.norm(e64)
    assert rc <= 1e-5 and re <= 1e-5, (rc, re)


@pytest.mark.gpu
def test_generic_path_matches_fused_and_oracle(oracle):
    """The generic kernels (spectral state in natural order) and the fused
    kernels compute the same step: both agree with the oracle to 1e-10."""
    p, c, e = active_landau(n=32, nvar=2, elastic=P.ELAST_HOMOG)
    q = p.copy()
    q.flags = P.FLAG_GENERIC
    o = oracle.OracleSim(p)
    o.set_fields(c, e)
    o.run(30)
    co, eo, _, _ = o.get_fields()
    for params in (p, q):
        with Simulation(params) as g:
            g.set_fields(c, e)
            g.timing(True)
            g.run(30)
            names = set(g.timing_report())
            cg, eg, _, _ = g.get_fields()
        assert ("lf_z_green_ch" in names) == (params.flags == 0)
        assert np.max(np.abs(cg - co)) <= TOL and np.max(np.abs(eg - eo)) <= TOL


@pytest.mark.gpu
def test_generic_path_fp32_error_after_1000_steps():
    """Accuracy of the generic FP32 path with spectral state (config-1 deck)."""
    from meumapps_ss_b200 import _lib
    from meumapps_ss_b200 import configs as CF
    w = CF.landau_config(1, precision=P.PREC_F64)
    c, e = _lib.init_uniform(128, 128, 128, 3, w.seed, w.c0, w.c_amp, w.eta_amp)
    out = {}
    for prec in (P.PREC_F64, P.PREC_F32):
        p = w.params.copy()
        p.precision = prec
        p.flags = P.FLAG_GENERIC
        with Simulation(p) as g:
            g.set_fields(c, e)
            g.run(1000, diag=False)
            out[prec] = g.get_fields()
    rc = np.linalg.norm(out[P.PREC_F32][0] - out[P.PREC_F64][0]) / np.linalg.norm(out[P.PREC_F64][0])
    re = np.linalg.norm(out[P.PREC_F32][1] - out[P.PREC_F64][1]) / np.linalg.norm(out[P.PREC_F64][1])
    assert rc <= 1e-5 and re <= 1e-5, (rc, re)
