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


# ------------------------------------------------------------------ error decks
# Inputs made on the host that drive the step into each of the reference's stops
# (ModFunc.f:55-67 through invert's rcond test; ModElastic.f:438-450 for the elastic
# divergence), with the status code the reference's err_flag would carry.
def singular_q_deck(n=16):
    """Stiffness without shear (C44 = 0): Q(k) = C_ijkl k_j k_l loses rank for k along
    an axis, so Omega(k) = Q^-1 does not exist (ModElastic.f:187, code 3).  The
    compliances stay those of a valid cubic medium: the C-ABI takes both as given."""
    p, c, e = active_landau(n, 1, elastic=P.ELAST_HOMOG)
    cs = CF.cubic(250.0, 150.0, 0.0)
    p.set_matrix("cela", 0, cs)
    p.set_matrix("cela", 1, cs)
    return p, c, e, 3


def singular_mix_deck(n=16):
    """Precipitate compliance -S (proportional factor -1) and h(eta) coupling: at eta = 0.5,
    h = 1/2 and the eldis mix h S_2 + (1 - h) S_1 = 0 (ModElastic.f:268-272, code 4)."""
    p, c, e = active_landau(n, 1, elastic=P.ELAST_HETERO, coupling=P.EIG_H)
    cm = CF.cubic(250.0, 150.0, 100.0)
    p.set_matrix("cela", 1, -cm)
    p.set_matrix("sela", 1, -np.linalg.inv(cm))
    e = e.copy()
    e[0, n // 2, n // 3, n // 4] = 0.5
    return p, c, e, 4


def singular_elener_deck(n=16):
    """Two variants with precipitate compliance S/2: where both order parameters are 1,
    h_1 + h_2 = 2, so eldis (matrix term only for sum h < 1) mixes 2 (S/2) = S, while
    elener, which always adds (1 - sum h) S_1 (ModElastic.f:597), gets S - S = 0 (code 6)."""
    p, c, e = active_landau(n, 2, elastic=P.ELAST_HETERO, coupling=P.EIG_H, ppt_scale=2.0)
    e = e.copy()
    e[:, n // 2, n // 2, n // 2] = 1.0
    return p, c, e, 6


def singular_z_deck(n=16):
    """KKS deck whose phases have zero curvature in their Gibbs parabolas: the constant
    rows of the interface-composition system (Multi_MEUMAPPS.f:426-448) vanish and the
    per-voxel Z solve is singular (Multi_MEUMAPPS.f:690, code 2)."""
    txt = CF.kks_input_txt(n, 1, 5, hetero=False)
    txt = txt.replace("2.0e4  0.0  0.10", "0.0  0.0  0.10").replace("2.0e4  -600.0  0.55", "0.0  -600.0  0.55")
    deck = P.parse_input_txt(txt)
    p = P.kks_params(deck)
    cons, phi = P.init_fields(deck)
    return p, cons, phi, 2


def diverging_elastic_deck(n=16):
    """Heterogeneous moduli with a precipitate ten times softer than the matrix: the
    fixed point diverges, the damping factor backtracks until newfac < 1e-7 and the
    step stops with ModElastic.f:446-450's trouble-converging exit (code 7)."""
    p, c, e = active_landau(n, 1, elastic=P.ELAST_HETERO, coupling=P.EIG_H, ppt_scale=0.1)
    return p, c, e, 7
