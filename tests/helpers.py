"""Shared builders for the tests (decks, seeded fields)."""
import numpy as np

from meumapps_ss_b200 import configs as CF
from meumapps_ss_b200 import params as P


def kks_case(n=16, nvar=1, steps=10, hetero=True, numel_in=2, nuc="single", radius=3, ny=None, nz=None):
    deck = P.parse_input_txt(CF.kks_input_txt(n, nvar, steps, hetero=hetero, numel_in=numel_in, nuc=nuc,
                                              radius=radius, ny=ny, nz=nz))
    p = P.kks_params(deck)
    cons, phi = P.init_fields(deck)
    return deck, p, cons, phi


def py_uniform(nx, ny, nz, nvar, seed, c0, c_amp, eta_amp):
    """Pure-Python restatement of the uniform-noise initialiser (small grids)."""
    r = P.Ran2(seed)
    n = nx * ny * nz
    c = np.empty(n)
    e = np.empty((nvar, n))
    for i in range(n):
        c[i] = c0 + c_amp * (2 * r() - 1)
        for v in range(nvar):
            e[v, i] = eta_amp * (2 * r() - 1)
    return c.reshape(1, nz, ny, nx), e.reshape(nvar, nz, ny, nx)


def active_landau(n=16, nvar=1, elastic=P.ELAST_HOMOG, precision=P.PREC_F64, coupling=P.EIG_ETA2, seed=-3,
                  dt=0.01, ppt_scale=1.0, cross_w=0.5, el_tol=1e-7):
    """A Landau deck that orders within a few hundred steps: c0 = 0.8 sits in
    the ordered region of the free energy and eta starts with +-0.5 noise."""
    eig = CF.tetragonal_variants(0.02, -0.005, nvar) if nvar > 1 else [[0.01, 0.01, 0.01]]
    p = CF.landau_params(n, nvar, eig, dt=dt, precision=precision, elastic=elastic, coupling=coupling,
                         ppt_scale=ppt_scale, cross_w=cross_w, el_tol=el_tol)
    c, e = py_uniform(n, n, n, nvar, seed, 0.8, 0.05, 0.5)
    return p, c, e
