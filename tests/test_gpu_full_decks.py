"""The plain FP64 path on full-size decks against the CPU FP64 oracle: deck 0
(64^3, one variant, 100 steps) and deck 1 (128^3, three variants, 20 steps),
both on the fused kernels, from the decks' own seeded initial fields.  The
gate is <= 1e-10 max-abs in c and eta over the run (checked at every chunk
boundary), with the fort.98 energies to 1e-9 relative."""
import numpy as np
import pytest

from meumapps_ss_b200 import configs as CF
from meumapps_ss_b200 import params as P
from meumapps_ss_b200.sim import Simulation

TOL = 1e-10


def _deck_parity(oracle, cfg, steps, chunks):
    w = CF.landau_config(cfg, precision=P.PREC_F64)
    p = w.params
    c, e = oracle.init_uniform(p.nx, p.ny, p.nz, p.nvar, w.seed, w.c0, w.c_amp, w.eta_amp)
    o = oracle.OracleSim(p)
    o.set_fields(c, e)
    worst = 0.0
    with Simulation(p) as g:
        g.set_fields(c, e)
        g.timing(True)
        for _ in range(chunks):
            do = o.run(steps // chunks)
            dg = g.run(steps // chunks)
            co, eo, _, _ = o.get_fields()
            cg, eg, _, _ = g.get_fields()
            worst = max(worst, np.max(np.abs(cg - co)), np.max(np.abs(eg - eo)))
            for k in ("fint", "fch", "elen", "etot"):
                rel = np.abs(dg[k] - do[k]) / np.maximum(np.abs(do[k]), 1e-30)
                assert np.max(rel) < 1e-9, k
        names = set(g.timing_report())
    assert "lf_z_green_ch" in names and "lf_plane_inv_stats_theta" in names
    return worst


@pytest.mark.gpu
def test_deck0_full_size_100_steps(oracle):
    assert _deck_parity(oracle, 0, 100, 4) <= TOL


@pytest.mark.gpu
def test_deck1_full_size_20_steps(oracle):
    assert _deck_parity(oracle, 1, 20, 2) <= TOL
