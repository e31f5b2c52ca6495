"""Host-side mirror of the reference's parameter set-up.

The reference reads ``Input.txt`` (Multi_MEUMAPPS.f:117-206), converts units and
fills its parameter module (Multi_MEUMAPPS.f:153-156, :218-236, :344-405 and
ModInitials.f:16-343).  In the drop-in deployment the Fortran driver keeps doing
that and copies the module variables into ``meu_params``; this module is the
same set-up written in Python so that the C-ABI can be driven without a Fortran
compiler (tests, benchmark, examples).

``MeuParams`` / ``MeuDiag`` mirror ``include/meu.h`` field for field.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math
from typing import Dict, List, Optional, Sequence

import numpy as np

MAX_VAR = 16
MAX_PH = 4
MAX_EL = 3
MAX_GP = 2 * MAX_EL + 1

MODEL_KKS = 0
MODEL_LANDAU = 1
PREC_F64 = 0
PREC_F32 = 1
ELAST_NONE = 0
ELAST_HOMOG = 1
ELAST_HETERO = 2
EIG_ETA2 = 0
EIG_H = 1
FLAG_GENERIC = 1
FLAG_AUTOTUNE = 2


class MeuParams(C.Structure):
    _fields_ = [
        ("step", C.c_int64),
        ("elastep0", C.c_int64),
        ("noise_step", C.c_int64),
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("model", C.c_int32),
        ("precision", C.c_int32),
        ("nvar", C.c_int32),
        ("numel", C.c_int32),
        ("numph", C.c_int32),
        ("nvar_ph", C.c_int32 * MAX_PH),
        ("elastic", C.c_int32),
        ("eig_coupling", C.c_int32),
        ("el_min_iter", C.c_int32),
        ("el_max_iter", C.c_int32),
        ("clip_phi", C.c_int32),
        ("diag_energy", C.c_int32),
        ("flags", C.c_int32),
        ("dt", C.c_double),
        ("b_mob", C.c_double),
        ("cmobs", C.c_double * MAX_EL),
        ("el_tol", C.c_double),
        ("e_mean", C.c_double * 6),
        ("grad_coeff", (C.c_double * 9) * MAX_VAR),
        ("trans_ppt", (C.c_double * 6) * MAX_VAR),
        ("cela", (C.c_double * 36) * MAX_PH),
        ("sela", (C.c_double * 36) * MAX_PH),
        ("gparams", (C.c_double * MAX_GP) * MAX_PH),
        ("wellph", C.c_double * MAX_PH),
        ("lan_a", C.c_double), ("lan_b", C.c_double), ("lan_c", C.c_double), ("lan_d", C.c_double),
        ("lan_c1", C.c_double), ("lan_c2", C.c_double), ("kappa_c", C.c_double), ("cross_w", C.c_double),
    ]

    # -- convenience views (column-major like the Fortran module arrays) --
    def set_matrix(self, name: str, index: int, mat: np.ndarray) -> None:
        arr = getattr(self, name)[index]
        flat = np.asarray(mat, dtype=np.float64).reshape(-1, order="F")
        for i, v in enumerate(flat):
            arr[i] = float(v)

    def matrix(self, name: str, index: int, n: int) -> np.ndarray:
        arr = getattr(self, name)[index]
        return np.array([arr[i] for i in range(n * n)], dtype=np.float64).reshape(n, n, order="F")

    def copy(self) -> "MeuParams":
        q = MeuParams()
        C.pointer(q)[0] = self
        return q


class MeuDiag(C.Structure):
    _fields_ = [
        ("step", C.c_int64),
        ("el_iters", C.c_int32),
        ("status", C.c_int32),
        ("fint", C.c_double), ("fw", C.c_double), ("fch", C.c_double), ("elen", C.c_double),
        ("etot", C.c_double),
        ("glob_min", C.c_double), ("glob_max", C.c_double), ("phi_max", C.c_double), ("solid", C.c_double),
        ("cmin", C.c_double), ("cmax", C.c_double), ("phimax", C.c_double), ("solid_now", C.c_double),
        ("cavg", C.c_double * MAX_EL),
    ]


DIAG_FIELDS = ["fint", "fw", "fch", "elen", "etot", "glob_min", "glob_max", "phi_max", "solid",
               "cmin", "cmax", "phimax", "solid_now"]


def diag_to_dict(rows: Sequence[MeuDiag]) -> Dict[str, np.ndarray]:
    out: Dict[str, np.ndarray] = {"step": np.array([r.step for r in rows]),
                                  "el_iters": np.array([r.el_iters for r in rows])}
    for f in DIAG_FIELDS:
        out[f] = np.array([getattr(r, f) for r in rows])
    out["cavg"] = np.array([[r.cavg[i] for i in range(MAX_EL)] for r in rows])
    return out


# ---------------------------------------------------------------- eltensor --
def eltensor(c: np.ndarray, cryst_type: int) -> np.ndarray:
    """Complete an elastic tensor from its independent constants
    (ModInitials.f:16-72)."""
    c = np.array(c, dtype=np.float64)
    if cryst_type == 1:  # cubic: C11, C12, C44
        c[0, 2] = c[0, 1]
        c[1, 1] = c[0, 0]
        c[1, 2] = c[0, 2]
        c[2, 2] = c[0, 0]
        c[4, 4] = c[3, 3]
        c[5, 5] = c[3, 3]
    if cryst_type == 2:  # tetragonal
        c[1, 1] = c[0, 0]
        c[4, 4] = c[3, 3]
        c[1, 2] = c[0, 2]
    if cryst_type == 3:  # hexagonal
        c[1, 1] = c[0, 0]
        c[1, 2] = c[0, 2]
        c[4, 4] = c[3, 3]
        c[5, 5] = 0.5 * (c[0, 0] - c[0, 1])
    if cryst_type == 4:  # trigonal
        c[1, 1] = c[0, 0]
        c[1, 2] = c[0, 2]
        c[1, 4] = -c[0, 4]
        c[3, 5] = -c[0, 4]
        c[4, 4] = c[3, 3]
        c[5, 5] = 0.5 * (c[0, 0] - c[0, 1])
    for j in range(1, 6):
        for i in range(j):
            c[j, i] = c[i, j]
    return c


def invert_checked(a: np.ndarray, flag: int) -> np.ndarray:
    """invert (ModFunc.f:44-72): inverse with the reciprocal-condition test
    rcond > 1e-16, else the error flag is raised."""
    a = np.asarray(a, dtype=np.float64)
    try:
        inv = np.linalg.inv(a)
    except np.linalg.LinAlgError:
        raise SetupError(flag, "singular matrix")
    rcond = 1.0 / (np.abs(a).sum(axis=0).max() * np.abs(inv).sum(axis=0).max())
    if not rcond > 1e-16:
        raise SetupError(flag, f"rcond={rcond}")
    return inv


class SetupError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"set-up error {code}: {msg}")
        self.code = code


# ------------------------------------------------------------- Input.txt --
class _Reader:
    """Fortran list-directed READ: every read starts on a new record and may
    continue onto following records until it has all its values."""

    def __init__(self, text: str):
        self.lines = text.splitlines()
        self.pos = 0

    @staticmethod
    def _tokens(line: str) -> List[str]:
        out, cur, quote = [], "", None
        for ch in line:
            if quote:
                if ch == quote:
                    quote = None
                else:
                    cur += ch
            elif ch in "'\"":
                quote = ch
            elif ch in " ,\t":
                if cur:
                    out.append(cur)
                    cur = ""
            elif ch == "/":
                break
            else:
                cur += ch
        if cur:
            out.append(cur)
        return out

    def read(self, n: int) -> List[str]:
        vals: List[str] = []
        while len(vals) < n:
            if self.pos >= len(self.lines):
                raise SetupError(100, "unexpected end of Input.txt")
            vals += self._tokens(self.lines[self.pos])
            self.pos += 1
        return vals[:n]


def _f(x: str) -> float:
    return float(x.replace("d", "e").replace("D", "e"))


@dataclasses.dataclass
class Deck:
    """Values read from Input.txt (Multi_MEUMAPPS.f:117-206)."""
    ndim: int
    dims: List[int]
    nx: int
    ny: int
    nz: int
    del_n: float
    nrun: int
    step: int
    elastep0: int
    nt: int
    t_step: float
    noise_step: int
    b_mob: float
    diff_coeff: float
    m_star: float
    sd: float
    noise: float
    ifreq: int
    nucstat: str
    targv: int
    vartot: int
    nmaxppt: int
    iseed: int
    var_lo: int
    var_hi: int
    radppt: List[int]
    addrad: List[int]
    disc_ener: float
    numph: int
    numel_in: int
    intfantiph: float
    e_mean: List[float]
    constat: str
    cav: List[float]
    cimax: List[float]
    cigrad: List[float]
    phi_init: float
    nvar: List[int]
    ctype: List[int]
    cela: List[np.ndarray]
    tstr: List[List[float]]
    eintf: List[List[float]]
    gparams: List[List[float]]


def parse_input_txt(text: str) -> Deck:
    r = _Reader(text)
    r.read(1)
    ndim, d1, d2 = (int(v) for v in r.read(3))
    r.read(1)
    vals = r.read(4)
    nx, ny, nz = (int(v) for v in vals[:3])
    del_n = _f(vals[3])
    v = r.read(6)
    nrun, step, elastep0, nt = int(v[0]), int(v[1]), int(v[2]), int(v[3])
    t_step, noise_step = _f(v[4]), int(v[5])
    b_mob, diff_coeff, m_star = (_f(x) for x in r.read(3))
    sd, noise = (_f(x) for x in r.read(2))
    ifreq = int(r.read(1)[0])
    r.read(1)
    v = r.read(5)
    nucstat, targv, vartot, nmaxppt, iseed = v[0], int(v[1]), int(v[2]), int(v[3]), int(v[4])
    var_lo, var_hi = (int(x) for x in r.read(2))
    radppt = [int(x) for x in r.read(3)]
    addrad = [int(x) for x in r.read(3)]
    disc_ener = _f(r.read(1)[0])
    r.read(1)
    numph, numel_in = (int(x) for x in r.read(2))
    intfantiph = _f(r.read(1)[0])
    e_mean = [_f(x) for x in r.read(3)]
    numel = numel_in - 1
    pmax = 2 * numel + 1
    r.read(1)
    constat = r.read(1)[0]
    cav, cimax, cigrad = [0.0] * numel, [0.0] * numel, [0.0] * numel
    for _ in range(numel):
        v = r.read(4)
        e = int(v[0]) - 1
        cav[e], cimax[e], cigrad[e] = _f(v[1]), _f(v[2]), _f(v[3])
    nvar = [0] * numph
    ctype = [0] * numph
    cela = [np.zeros((6, 6)) for _ in range(numph)]
    tstr = [[0.0] * 3 for _ in range(numph)]
    eintf = [[0.0] * 3 for _ in range(numph)]
    gp = [[0.0] * pmax for _ in range(numph)]
    r.read(1)
    phi_init = _f(r.read(1)[0])
    v = r.read(3)
    n = int(v[0]) - 1
    nvar[n], ctype[n] = int(v[1]), int(v[2])
    c11, c12, c44 = (_f(x) for x in r.read(3))
    cela[n][0, 0], cela[n][0, 1], cela[n][3, 3] = c11, c12, c44
    gp[n] = [_f(x) for x in r.read(pmax)]
    for i in range(2, numph + 1):
        r.read(1)
        v = r.read(3)
        n = int(v[0]) - 1
        nvar[n], ctype[n] = int(v[1]), int(v[2])
        if ctype[n] == 1:
            c11, c12, c44 = (_f(x) for x in r.read(3))
            cela[n][0, 0], cela[n][0, 1], cela[n][3, 3] = c11, c12, c44
        else:
            a = [_f(x) for x in r.read(6)]
            cela[n][0, 0], cela[n][0, 1], cela[n][0, 2], cela[n][1, 1], cela[n][1, 2], cela[n][2, 2] = a
            a = [_f(x) for x in r.read(6)]
            cela[n][3, 3], cela[n][3, 4], cela[n][3, 5], cela[n][4, 4], cela[n][4, 5], cela[n][5, 5] = a
        tstr[n] = [_f(x) for x in r.read(3)]
        eintf[n] = [_f(x) for x in r.read(3)]
        gp[n] = [_f(x) for x in r.read(pmax)]
        if i != n + 1:
            raise SetupError(4, "phase numbering")
    if vartot + 1 - sum(nvar) != 0:
        raise SetupError(1, "variant numbers")
    return Deck(ndim, [d1, d2], nx, ny, nz, del_n, nrun, step, elastep0, nt, t_step, noise_step, b_mob,
                diff_coeff, m_star, sd, noise, ifreq, nucstat, targv, vartot, nmaxppt, iseed, var_lo, var_hi,
                radppt, addrad, disc_ener, numph, numel_in, intfantiph, e_mean, constat, cav, cimax, cigrad,
                phi_init, nvar, ctype, cela, tstr, eintf, gp)


def _zhou_q() -> np.ndarray:
    """Rotation to the delta habit plane (ModInitials.f:219-229)."""
    q = np.zeros((3, 3))
    s2, s3, s6 = math.sqrt(2.0), math.sqrt(3.0), math.sqrt(6.0)
    q[0, 0], q[1, 0], q[2, 0] = 1.0 / s2, 0.0, -1.0 / s2
    q[0, 1], q[1, 1], q[2, 1] = 1.0 / s3, 1.0 / s3, 1.0 / s3
    q[0, 2], q[1, 2], q[2, 2] = 1.0 / s6, -2.0 / s6, 1.0 / s6
    return q


def kks_params(deck: Deck, precision: int = PREC_F64, sym_var: Optional[Sequence[np.ndarray]] = None,
               myid: int = 0) -> MeuParams:
    """Set-up of Multi_MEUMAPPS.f:153-405 (+ ModInitials InitElasticMat,
    InitTransGrad) producing the parameter block of the step."""
    p = MeuParams()
    numel = deck.numel_in - 1
    numph = deck.numph
    if numel > MAX_EL or numph > MAX_PH or deck.vartot > MAX_VAR:
        raise SetupError(100, "deck exceeds the compiled limits")
    p.model = MODEL_KKS
    p.precision = precision
    p.nx, p.ny, p.nz = deck.nx, deck.ny, deck.nz
    p.nvar, p.numel, p.numph = deck.vartot, numel, numph
    for i in range(numph):
        p.nvar_ph[i] = deck.nvar[i]
    p.step, p.elastep0, p.noise_step = deck.step, deck.elastep0, deck.noise_step
    p.elastic = ELAST_HETERO
    p.el_min_iter, p.el_max_iter, p.el_tol = 4, 10, 1e-7
    p.clip_phi = 1
    p.diag_energy = 1
    p.dt, p.b_mob = deck.t_step, deck.b_mob
    for i in range(3):
        p.e_mean[i] = deck.e_mean[i]
    # Gparams / molar volume; 1.055e-5 is a REAL*4 literal (:221, :225)
    mv = float(np.float32(1.055e-5))
    gp = [list(g) for g in deck.gparams]
    for n in range(numph):
        for e in range(numel + 1):
            gp[n][e] = gp[n][e] / mv
    for e in range(numel):
        gp[0][e] = gp[0][e] + deck.disc_ener
    for n in range(numph):
        for j in range(2 * numel + 1):
            p.gparams[n][j] = gp[n][j]
    # InitElasticMat (ModInitials.f:76-116)
    for n in range(numph):
        c = deck.cela[n]
        if c[0, 0] <= 0:
            p.set_matrix("cela", n, np.zeros((6, 6)))
            p.set_matrix("sela", n, np.zeros((6, 6)))
        else:
            cf = eltensor(c, deck.ctype[n])
            p.set_matrix("cela", n, cf)
            p.set_matrix("sela", n, invert_checked(cf, 20))
    # interface width, wells, variants (Multi_MEUMAPPS.f:354-376)
    b_width = 5.0 * deck.del_n
    sume = [sum(e) for e in deck.eintf]
    trans = np.zeros((6, MAX_VAR))
    grad = np.zeros((3, 3, MAX_VAR))
    ivn = 0
    for nphc in range(2, numph + 1):
        p.wellph[nphc - 1] = 6.0 * sume[nphc - 1] / b_width
        ivn += deck.nvar[nphc - 2]
        _init_trans_grad(deck, nphc, ivn, b_width, trans, grad, sym_var)
    p.wellph[0] = 6.0 * deck.intfantiph / b_width
    grad /= deck.del_n * deck.del_n
    for v in range(deck.vartot):
        for i in range(6):
            p.trans_ppt[v][i] = trans[i, v]
        g = grad[:, :, v].reshape(-1, order="F")
        for i in range(9):
            p.grad_coeff[v][i] = g[i]
    for e in range(numel):
        p.cmobs[e] = deck.diff_coeff / (deck.del_n * deck.del_n)
    return p


def _init_trans_grad(deck: Deck, nphc: int, i0: int, b_width: float, trans: np.ndarray, grad: np.ndarray,
                     sym_var: Optional[Sequence[np.ndarray]]) -> None:
    """InitTransGrad (ModInitials.f:122-343); i0 is the 1-based first variant."""
    nv = deck.nvar[nphc - 1]
    e = deck.eintf[nphc - 1]
    t = deck.tstr[nphc - 1]
    a = i0 - 1
    if nv == 1:
        trans[0:3, a] = t
        for d in range(3):
            grad[d, d, a] = b_width * e[d]
    if nv == 3:
        trans[0:3, a] = [t[0], t[1], t[2]]
        trans[0:3, a + 1] = [t[1], t[0], t[2]]
        trans[0:3, a + 2] = [t[1], t[2], t[0]]
        for v in range(a, a + 3):
            for d in range(3):
                grad[d, d, v] = b_width * e[d]
    if nv == 12:
        if sym_var is None or len(sym_var) < 12:
            raise SetupError(2, "sym_var.inp does not exist")
        q = _zhou_q()
        A = np.diag([b_width * e[0], b_width * e[1], b_width * e[2]])
        A = (q @ A) @ q.T
        B = np.diag(t)
        B = (q @ B) @ q.T
        for k, v in enumerate(range(a, a + 12)):
            sym = np.asarray(sym_var[k], dtype=np.float64)
            grad[:, :, v] = (sym.T @ A) @ sym
            bp = (sym.T @ B) @ sym
            trans[:, v] = [bp[0, 0], bp[1, 1], bp[2, 2], bp[1, 2], bp[0, 2], bp[0, 1]]


# ----------------------------------------------------------- layouts --
def to_fortran(soa: np.ndarray) -> np.ndarray:
    """(ncomp, nz, ny, nx) SoA -> flat Fortran array A(ncomp,Nx,Ny,Nz)
    (component index fastest)."""
    soa = np.asarray(soa, dtype=np.float64)
    return np.ascontiguousarray(np.moveaxis(soa, 0, -1)).reshape(-1)


def from_fortran(flat: np.ndarray, ncomp: int, nx: int, ny: int, nz: int) -> np.ndarray:
    a = np.asarray(flat, dtype=np.float64).reshape(nz, ny, nx, ncomp)
    return np.ascontiguousarray(np.moveaxis(a, -1, 0))


# ---------------------------------------------------------- ran_2 (host) --
class Ran2:
    """ran_2.f:1-42 with its SAVE state as attributes (bit-exact; Python ints)."""
    IM1, IM2 = 2147483563, 2147483399
    IMM1 = IM1 - 1
    IA1, IA2, IQ1, IQ2, IR1, IR2 = 40014, 40692, 53668, 52774, 12211, 3791
    NTAB = 32
    NDIV = 1 + IMM1 // NTAB
    AM = float(np.float32(1.0) / np.float32(IM1))
    RNMX = 1.0 - 1.2e-7

    def __init__(self, iseed: int):
        self.idum = int(iseed)
        self.idum2 = 123456789
        self.iy = 0
        self.iv = [0] * self.NTAB

    @staticmethod
    def _div(a: int, b: int) -> int:  # Fortran integer division truncates toward zero
        q = abs(a) // abs(b)
        return q if (a >= 0) == (b >= 0) else -q

    def __call__(self) -> float:
        if self.idum <= 0:
            self.idum = max(-self.idum, 1)
            self.idum2 = self.idum
            for j in range(self.NTAB + 8, 0, -1):
                k = self._div(self.idum, self.IQ1)
                self.idum = self.IA1 * (self.idum - k * self.IQ1) - k * self.IR1
                if self.idum < 0:
                    self.idum += self.IM1
                if j <= self.NTAB:
                    self.iv[j - 1] = self.idum
            self.iy = self.iv[0]
        k = self._div(self.idum, self.IQ1)
        self.idum = self.IA1 * (self.idum - k * self.IQ1) - k * self.IR1
        if self.idum < 0:
            self.idum += self.IM1
        k = self._div(self.idum2, self.IQ2)
        self.idum2 = self.IA2 * (self.idum2 - k * self.IQ2) - k * self.IR2
        if self.idum2 < 0:
            self.idum2 += self.IM2
        j = 1 + self._div(self.iy, self.NDIV)
        self.iy = self.iv[j - 1] - self.idum2
        self.iv[j - 1] = self.idum
        if self.iy < 1:
            self.iy += self.IMM1
        return min(self.AM * self.iy, self.RNMX)


def init_fields(deck: Deck, ran: Optional[Ran2] = None):
    """InitFields (ModInitials.f:415-678) for one rank: returns SoA
    (cons[numel], phi[vartot]) arrays of shape (n, nz, ny, nx)."""
    numel = deck.numel_in - 1
    nx, ny, nz = deck.nx, deck.ny, deck.nz
    phi = np.full((deck.vartot, nz, ny, nx), deck.phi_init)
    cons = np.empty((numel, nz, ny, nx))
    for e in range(numel):
        cons[e] = deck.cav[e]
    mnx, mny, mnz = nx // 2, ny // 2, nz // 2
    r0 = deck.radppt[0] ** 2 + deck.radppt[1] ** 2 + deck.radppt[2] ** 2
    nuc = deck.nucstat.strip()
    targv = deck.targv
    if nuc == "single":
        if targv == 0:
            targv = 1
        rp = deck.radppt
        for k in range(-rp[2], rp[2] + 1):
            for j in range(-rp[1], rp[1] + 1):
                for i in range(-rp[0], rp[0] + 1):
                    s = (float(i) / rp[0]) ** 2 + (float(j) / rp[1]) ** 2 + (float(k) / rp[2]) ** 2
                    if s <= 1.0:
                        ii, jj, kk = i + mnx, j + mny, k + mnz
                        if 1 <= ii <= nx and 1 <= jj <= ny and 1 <= kk <= nz:
                            phi[targv - 1, kk - 1, jj - 1, ii - 1] = 1.0
    elif nuc == "random":
        ran = ran or Ran2(deck.iseed)
        for k in range(nz):
            for j in range(ny):
                for i in range(nx):
                    rv = int(ran() * deck.vartot + 1.0)
                    phi[rv - 1, k, j, i] = float(np.float32(0.1))
    elif nuc == "multiple":
        ran = ran or Ran2(deck.iseed)
        zz, yy, xx = np.meshgrid(np.arange(1, nz + 1), np.arange(1, ny + 1), np.arange(1, nx + 1), indexing="ij")
        nppt = 1
        while nppt <= deck.nmaxppt:
            while True:
                ix = int(ran() * nx + 1.0)
                jy = int(ran() * ny + 1.0)
                kz = int(ran() * nz + 1.0)
                if targv == 0:
                    rv = int(deck.var_lo + ran() * (deck.var_hi - deck.var_lo) + 1.0)
                else:
                    rv = targv
                rd = (xx - ix) ** 2 + (yy - jy) ** 2 + (zz - kz) ** 2
                inside = rd <= r0
                if not np.any(inside[None, ...] & (phi > 0.0)):
                    break
            phi[rv - 1][inside] = 1.0
            nppt += 1
    if deck.constat.strip() == "cppt" and targv >= 1:
        mask = phi[targv - 1] > 0.9
        for e in range(numel):
            cons[e][mask] = deck.cimax[e]
    return cons, phi
