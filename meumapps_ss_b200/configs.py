"""Workload decks.

* ``kks_input_txt`` writes a deck in the reference's own ``Input.txt`` format
  (read by Multi_MEUMAPPS.f:117-206 and by ``params.parse_input_txt``); the
  reference ships no example input, so these decks are synthetic: a binary
  alloy (one solute), one matrix and one precipitate phase with 1 or 3
  variants, heterogeneous cubic moduli and a spherical nucleus.
* ``ensemble_config`` draws the members of the batched ensemble (configuration 3).
* ``landau_params`` / ``landau_config`` build the Landau decks (one conserved
  concentration c, p non-conserved order parameters eta).  Their free energy
  is not in the reference; it uses the reference's spectral skeleton and
  elasticity (see include/meu.h for the functional).
"""
from __future__ import annotations

import dataclasses
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import params as P


def kks_input_txt(n: int = 16, nvar: int = 1, steps: int = 10, hetero: bool = True, elastep0: int = 1,
                  radius: int = 3, t_step: float = 1.0e-3, noise_step: int = 0, nuc: str = "single",
                  numel_in: int = 2, ny: Optional[int] = None, nz: Optional[int] = None) -> str:
    ny = ny or n
    nz = nz or n
    pmax = 2 * (numel_in - 1) + 1
    # Gparams rows per phase: curvature(s), constant, equilibrium composition(s) (J/mol)
    if numel_in == 2:
        gm = "2.0e4  0.0  0.10"
        gp = "2.0e4  -600.0  0.55"
        conc = "1  0.15  0.55  0.0"
    else:
        gm = "2.0e4 1.5e4  0.0  0.10 0.05"
        gp = "2.0e4 1.8e4  -600.0  0.55 0.20"
        conc = "1  0.15  0.55  0.0\n2  0.07  0.20  0.0"
    assert len(gm.split()) == pmax
    tstr = "0.010 0.010 0.005" if nvar == 1 else "0.020 -0.005 -0.005"
    cppt = "1.80e11 1.00e11 0.50e11" if hetero else "1.60e11 0.90e11 0.45e11"
    return f"""MPI
1 1 1
simulation
{n} {ny} {nz} 1.0e-9
1 1 {elastep0} {steps} {t_step} {noise_step}
2.0e-8 1.0e-16 1.0
1.0e-3 0.0
1000
nucleation
{nuc} 1 {nvar} 3 -5
1 {nvar}
{radius} {radius} {radius}
1 1 1
0.0
phases
2 {numel_in}
0.10
0.0 0.0 0.0
concentration
cppt
{conc}
matrix
0.0
1 1 1
1.60e11 0.90e11 0.45e11
{gm}
precipitate
2 {nvar} 1
{cppt}
{tstr}
0.10 0.10 0.10
{gp}
"""


def tetrahedral_rotations() -> List[np.ndarray]:
    """The 12 proper rotations of the tetrahedral group (identity, three 180 degree
    turns about the cube axes, eight 120 degree turns about the body diagonals),
    as the 12 orientation matrices a `sym_var.inp` file lists for 12-variant KKS
    decks (read at ModInitials.f:200-338).  The reference ships no such file."""
    rots = [np.eye(3)]
    for ax in range(3):
        m = -np.eye(3)
        m[ax, ax] = 1.0
        rots.append(m)
    for sx in (1, -1):
        for sy in (1, -1):
            d = np.array([1.0, sx, sy]) / np.sqrt(3.0)
            for ang in (2 * np.pi / 3, -2 * np.pi / 3):
                k = np.array([[0, -d[2], d[1]], [d[2], 0, -d[0]], [-d[1], d[0], 0]])
                r = np.eye(3) + np.sin(ang) * k + (1 - np.cos(ang)) * (k @ k)
                rots.append(np.round(r, 15))
    return rots


def cubic(c11: float, c12: float, c44: float) -> np.ndarray:
    c = np.zeros((6, 6))
    c[0, 0], c[0, 1], c[3, 3] = c11, c12, c44
    return P.eltensor(c, 1)


def landau_params(n: int, nvar: int, eig: Sequence[Sequence[float]], *, coupling: int = P.EIG_ETA2,
                  elastic: int = P.ELAST_HOMOG, dt: float = 0.01, precision: int = P.PREC_F64,
                  A: float = 2.0, B: float = 1.0, Cq: float = 1.0, D: float = 1.0, c1: float = 0.05,
                  c2: float = 0.95, kappa_c: float = 1.0, kappa_eta: float = 1.0, M: float = 1.0,
                  L: float = 1.0, cross_w: float = 0.0, moduli: Tuple[float, float, float] = (250.0, 150.0, 100.0),
                  ppt_scale: float = 1.0, el_tol: float = 1e-7, el_min_iter: int = 4, el_max_iter: int = 10,
                  diag_energy: int = 1, ny: Optional[int] = None, nz: Optional[int] = None) -> P.MeuParams:
    p = P.MeuParams()
    p.model = P.MODEL_LANDAU
    p.precision = precision
    p.nx, p.ny, p.nz = n, ny or n, nz or n
    p.nvar, p.numel, p.numph = nvar, 1, 2
    p.nvar_ph[0], p.nvar_ph[1] = 1, nvar
    p.step, p.elastep0, p.noise_step = 1, 1, 0
    p.elastic = elastic
    p.eig_coupling = coupling
    p.el_min_iter, p.el_max_iter, p.el_tol = el_min_iter, el_max_iter, el_tol
    p.clip_phi = 0
    p.diag_energy = diag_energy
    p.dt, p.b_mob = dt, L
    p.cmobs[0] = M
    cm = cubic(*moduli)
    p.set_matrix("cela", 0, cm)
    p.set_matrix("sela", 0, np.linalg.inv(cm))
    cp = cm * ppt_scale
    p.set_matrix("cela", 1, cp)
    p.set_matrix("sela", 1, np.linalg.inv(cp))
    for v in range(nvar):
        e = list(eig[v]) + [0.0] * (6 - len(eig[v]))
        for i in range(6):
            p.trans_ppt[v][i] = e[i]
        g = (kappa_eta * np.eye(3)).reshape(-1, order="F")
        for i in range(9):
            p.grad_coeff[v][i] = g[i]
    p.lan_a, p.lan_b, p.lan_c, p.lan_d = A, B, Cq, D
    p.lan_c1, p.lan_c2 = c1, c2
    p.kappa_c = kappa_c
    p.cross_w = cross_w
    return p


def tetragonal_variants(mag_a: float, mag_b: float, count: int) -> List[List[float]]:
    base = [[mag_a, mag_b, mag_b], [mag_b, mag_a, mag_b], [mag_b, mag_b, mag_a]]
    return [base[i % 3] for i in range(count)]


@dataclasses.dataclass
class Workload:
    name: str
    params: P.MeuParams
    steps: int
    seed: int
    c0: float
    c_amp: float
    eta_amp: float


def landau_config(k: int, n: Optional[int] = None, precision: int = P.PREC_F32) -> Workload:
    """Configurations 0-2 of the Landau decks (sizes overridable for tests).

    0: 64^3, 1 eta, dilatational eps0 = 0.01 eta^2 I, dt 0.01, FP64, seed -1.
    1: 128^3, 3 tetragonal variants diag(0.02,-0.005,-0.005) and permutations,
       cross-term weight 0.5, dt 0.005, c0 = 0.2 +- 0.01, seed -7.
    2: 512^3, 4 variants 0.015*diag(1,-1/4,-1/4) (+ permutations, v4 = v1),
       precipitate moduli 1.5x, h(eta) coupling, heterogeneous fixed point to
       1e-8, dt 0.005, noise +-0.005, seed -11.
    Positive seeds of the decks are negated: ran_2 initialises only for idum <= 0.
    """
    if k == 0:
        n = n or 64
        p = landau_params(n, 1, [[0.01, 0.01, 0.01]], dt=0.01, precision=precision)
        return Workload("landau-cfg0-64^3-1var-homog", p, 1000, -1, 0.15, 0.01, 0.001)
    if k == 1:
        n = n or 128
        p = landau_params(n, 3, tetragonal_variants(0.02, -0.005, 3), dt=0.005, cross_w=0.5,
                          precision=precision)
        return Workload("landau-cfg1-128^3-3var-homog", p, 5000, -7, 0.2, 0.01, 0.001)
    if k == 2:
        n = n or 512
        p = landau_params(n, 4, tetragonal_variants(0.015, -0.015 / 4, 4), dt=0.005, cross_w=0.5,
                          coupling=P.EIG_H, elastic=P.ELAST_HETERO, ppt_scale=1.5, el_tol=1e-8,
                          precision=precision)
        return Workload("landau-cfg2-512^3-4var-hetero", p, 500, -11, 0.2, 0.01, 0.005)
    raise ValueError(k)


def adjoint_config(n: int = 128, precision: int = P.PREC_F32, kappa: float = 1.0, L: float = 1.0, M: float = 1.0,
                   eps0: float = 0.01) -> Workload:
    """Configuration 4: the configuration-0 deck (one eta and c, homogeneous cubic
    elasticity, dilatational eps0 eta^2 I, dt 0.01, c = 0.15 +- 0.01,
    eta +- 0.001, seed -1) on an n^3 grid for 200 steps with gradient
    parameters kappa (kappa_c = kappa_eta), L, M and eps0.  The calibration
    target is the FP64 forward at kappa 1.2, L 0.8, M 1.1, eps0 0.012."""
    p = landau_params(n, 1, [[eps0, eps0, eps0]], dt=0.01, precision=precision, kappa_c=kappa, kappa_eta=kappa,
                      M=M, L=L)
    return Workload(f"landau-adjoint-{n}^3-1var", p, 200, -1, 0.15, 0.01, 0.001)


ADJOINT_TARGET = dict(kappa=1.2, L=0.8, M=1.1, eps0=0.012)
ADJOINT_START = dict(kappa=1.0, L=1.0, M=1.0, eps0=0.01)
ADJOINT_CHECKPOINT_EVERY = 20


ENSEMBLE_SIZES = (32, 48, 64, 96, 128)


def ensemble_config(count: int = 96, precision: int = P.PREC_F32, sizes: Sequence[int] = ENSEMBLE_SIZES,
                    draw_seed: int = -3) -> List[Workload]:
    """Configuration 3: ``count`` independent single-variant runs of the
    configuration-0 deck.  Member m (seed -(m+1)) draws, with ran_2 seeded by
    ``draw_seed``, its grid uniformly from ``sizes`` and B ~ U(0.5, 1.5),
    eps0 ~ U(0.005, 0.02) (dilatational eps0 eta^2 I), c0 ~ U(0.1, 0.3); c noise
    +-0.01, eta noise +-0.001, dt 0.01, 2000 steps."""
    r = P.Ran2(draw_seed)
    out = []
    for m in range(count):
        n = sizes[min(int(r() * len(sizes)), len(sizes) - 1)]
        b = 0.5 + r()
        e0 = 0.005 + 0.015 * r()
        c0 = 0.1 + 0.2 * r()
        p = landau_params(n, 1, [[e0, e0, e0]], dt=0.01, precision=precision, B=b)
        out.append(Workload(f"landau-ens-{m}-{n}^3", p, 2000, -(m + 1), c0, 0.01, 0.001))
    return out


def uniform_fields(w: Workload) -> Tuple[np.ndarray, np.ndarray]:
    """Seeded uniform-noise initial fields (SoA float64) drawn with ran_2 in
    Fortran order: per voxel c then eta_1..eta_p."""
    from . import _lib
    p = w.params
    return _lib.init_uniform(p.nx, p.ny, p.nz, p.nvar, w.seed, w.c0, w.c_amp, w.eta_amp)
