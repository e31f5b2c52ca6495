"""ctypes binding of the CPU FP64 oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline / reference arm of bench.py.  Parity status: unpinned by
reference artefacts (the reference ships none and its Fortran build is not
compilable here).  Pinned on the CPU against numpy.fft (tests/test_oracle_fft.py),
known answers -- single-mode decay, uniform fields, mass conservation,
Khachaturyan's closed-form inclusion energy (Landau, and the KKS model's eldis +
elener with equal moduli) -- a numpy restatement of one KKS step of the reference
(tests/test_oracle_kks_mirror.py) and a numpy restatement of one
Landau step (tests/test_oracle_kat.py).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional, Tuple

import numpy as np

from meumapps_ss_b200 import params as P

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        src = os.path.join(_HERE, "meu_oracle.c")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            build()
        L = C.CDLL(path)
        vp, dp = C.c_void_p, C.POINTER(C.c_double)
        L.orc_create.restype = vp
        L.orc_create.argtypes = [C.POINTER(P.MeuParams)]
        L.orc_destroy.argtypes = [vp]
        L.orc_set_fields.argtypes = [vp, dp, dp, dp]
        L.orc_get_fields.argtypes = [vp, dp, dp, dp, dp]
        L.orc_add_noise.argtypes = [vp, dp]
        L.orc_run.argtypes = [vp, C.c_int, C.POINTER(P.MeuDiag)]
        L.orc_get_step.restype = C.c_int64
        L.orc_get_step.argtypes = [vp]
        L.orc_last_iters.argtypes = [vp]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_rfft3.argtypes = [C.c_int, C.c_int, C.c_int, dp, dp]
        L.orc_irfft3.argtypes = [C.c_int, C.c_int, C.c_int, dp, dp]
        L.orc_invert.argtypes = [dp, C.c_int]
        L.orc_ran2.restype = C.c_double
        L.orc_ran2.argtypes = [C.c_void_p]
        L.orc_ran2_init.argtypes = [C.c_void_p, C.c_int32]
        L.orc_langevin.restype = C.c_double
        L.orc_langevin.argtypes = [C.c_void_p, C.c_double]
        L.orc_init_uniform.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                       C.c_double, dp, dp]
        _LIB = L
    return _LIB


def _dp(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def get_threads() -> int:
    return int(lib().orc_get_threads())


def rfft3(x: np.ndarray) -> np.ndarray:
    """f_trans: x of shape (nz, ny, nx) -> (nz, ny, nx//2+1), scaled 1/N."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    nz, ny, nx = x.shape
    out = np.empty((nz, ny, nx // 2 + 1), dtype=np.complex128)
    lib().orc_rfft3(nx, ny, nz, _dp(x), out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def irfft3(k: np.ndarray, nx: int) -> np.ndarray:
    k = np.ascontiguousarray(k, dtype=np.complex128)
    nz, ny, _ = k.shape
    out = np.empty((nz, ny, nx), dtype=np.float64)
    lib().orc_irfft3(nx, ny, nz, k.ctypes.data_as(C.POINTER(C.c_double)), _dp(out))
    return out


def invert(a: np.ndarray) -> Tuple[int, np.ndarray]:
    m = np.asfortranarray(a, dtype=np.float64).copy(order="F")
    st = lib().orc_invert(m.ctypes.data_as(C.POINTER(C.c_double)), m.shape[0])
    return st, m


class Ran2State(C.Structure):
    _fields_ = [("idum", C.c_int32), ("idum2", C.c_int32), ("iy", C.c_int32), ("iv", C.c_int32 * 32)]


class OracleRan2:
    def __init__(self, iseed: int):
        self.s = Ran2State()
        lib().orc_ran2_init(C.byref(self.s), int(iseed))

    def __call__(self) -> float:
        return lib().orc_ran2(C.byref(self.s))

    def langevin(self, sd: float) -> float:
        return lib().orc_langevin(C.byref(self.s), float(sd))


def init_uniform(nx: int, ny: int, nz: int, nvar: int, seed: int, c0: float, c_amp: float,
                 eta_amp: float) -> Tuple[np.ndarray, np.ndarray]:
    """Uniform-noise initial fields drawn with the oracle's own ran_2 (SoA float64:
    (1,nz,ny,nx), (nvar,nz,ny,nx))."""
    s = Ran2State()
    lib().orc_ran2_init(C.byref(s), int(seed))
    n3 = nx * ny * nz
    cons = np.empty(n3)
    phi = np.empty(n3 * nvar)
    lib().orc_init_uniform(C.byref(s), nx, ny, nz, nvar, c0, c_amp, eta_amp, _dp(cons), _dp(phi))
    return cons.reshape(1, nz, ny, nx), P.from_fortran(phi, nvar, nx, ny, nz)


class OracleSim:
    """FP64 CPU restatement with the same life cycle as the C-ABI handle.
    Fields are structure-of-arrays (ncomp, nz, ny, nx)."""

    def __init__(self, p: P.MeuParams):
        self.p = p.copy()
        self.h = lib().orc_create(C.byref(self.p))
        if not self.h:
            raise MemoryError("orc_create failed")
        self.shape = (p.nz, p.ny, p.nx)

    def close(self) -> None:
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def set_fields(self, cons: np.ndarray, phi: np.ndarray, ustate: Optional[np.ndarray] = None) -> None:
        c = np.ascontiguousarray(cons, dtype=np.float64)
        f = np.ascontiguousarray(phi, dtype=np.float64)
        u = None if ustate is None else np.ascontiguousarray(ustate, dtype=np.float64)
        lib().orc_set_fields(self.h, _dp(c), _dp(f), _dp(u))

    def add_noise(self, incr: np.ndarray) -> None:
        a = np.ascontiguousarray(incr, dtype=np.float64)
        lib().orc_add_noise(self.h, _dp(a))

    def run(self, nsteps: int):
        rows = (P.MeuDiag * max(nsteps, 1))()
        st = lib().orc_run(self.h, int(nsteps), rows)
        if st:
            raise RuntimeError(f"oracle step failed with status {st}")
        return P.diag_to_dict(list(rows)[:nsteps])

    def get_fields(self):
        p = self.p
        n = (p.nz, p.ny, p.nx)
        cons = np.empty((p.numel,) + n)
        phi = np.empty((p.nvar,) + n)
        el = np.empty(n)
        u = np.empty((12,) + n)
        lib().orc_get_fields(self.h, _dp(cons), _dp(phi), _dp(el), _dp(u))
        return cons, phi, el, u

    @property
    def step(self) -> int:
        return int(lib().orc_get_step(self.h))
