"""Loader of the in-tree ``libmeu.so`` (the C-ABI of include/meu.h).

The product path has no fallback: if the shared library is missing or was
built from older sources, ``lib()`` raises instead of computing anything on
the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
import re
from typing import List, Tuple

import numpy as np

from . import params as P

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmeu.so")
HEADER = os.path.join(HERE, "..", "include", "meu.h")
_LIB = None


class MeuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"meu error {code}: {msg}")
        self.code = code


class Ran2State(C.Structure):
    _fields_ = [("idum", C.c_int32), ("idum2", C.c_int32), ("iy", C.c_int32), ("iv", C.c_int32 * 32)]


def header_functions() -> List[str]:
    """Names of every function declared in include/meu.h."""
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(meu_[a-z_0-9]+)\s*\(", txt, flags=re.M)


def lib():
    """Load libmeu.so; raise if it is absent (no CPU fallback exists)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise MeuError(101, f"{LIB_PATH} is missing: build it with `python -m meumapps_ss_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, dp, i32, i64 = C.c_void_p, C.POINTER(C.c_double), C.c_int32, C.c_int64
    L.meu_create.argtypes = [C.POINTER(P.MeuParams), C.POINTER(vp)]
    L.meu_set_fields.argtypes = [vp, dp, dp, dp]
    L.meu_add_noise.argtypes = [vp, dp]
    L.meu_run.argtypes = [vp, i32, C.POINTER(P.MeuDiag)]
    L.meu_run_noise.argtypes = [vp, i32, C.POINTER(Ran2State), C.c_double, C.POINTER(P.MeuDiag)]
    L.meu_get_fields.argtypes = [vp, dp, dp, dp, dp]
    L.meu_get_step.argtypes = [vp]
    L.meu_get_step.restype = i64
    L.meu_last_error.argtypes = [vp]
    L.meu_last_error.restype = C.c_char_p
    L.meu_destroy.argtypes = [vp]
    L.meu_ran2_init.argtypes = [C.POINTER(Ran2State), i32]
    L.meu_ran2.argtypes = [C.POINTER(Ran2State)]
    L.meu_ran2.restype = C.c_double
    L.meu_langevin.argtypes = [C.POINTER(Ran2State), C.c_double]
    L.meu_langevin.restype = C.c_double
    L.meu_langevin_fill.argtypes = [C.POINTER(Ran2State), C.c_double, i64, dp, i32]
    L.meu_init_uniform.argtypes = [C.POINTER(Ran2State), i32, i32, i32, i32, C.c_double, C.c_double, C.c_double, dp, dp]
    L.meu_params_from_gparams.argtypes = [i32, i32, i32, i32, i32, i32, C.POINTER(C.c_int32), i64, i64, i64,
                                          C.c_double, C.c_double, dp, dp, dp, dp, dp, dp, dp, dp,
                                          C.POINTER(P.MeuParams)]
    L.meu_fft_roundtrip.argtypes = [i32, i32, i32, i32, dp, dp, dp]
    L.meu_fft_roundtrip_noalloc.argtypes = [i32, i32, i32, i32, vp, vp, vp]
    L.meu_slab_fft_create.argtypes = [i32, i32, i32, i32, i32, i32, C.POINTER(vp)]
    L.meu_slab_fft_sizes.argtypes = [vp, C.POINTER(i64)]
    L.meu_slab_fft_forward_planes.argtypes = [vp, vp, vp, vp]
    L.meu_slab_fft_forward_columns.argtypes = [vp, vp, vp]
    L.meu_slab_fft_inverse_columns.argtypes = [vp, vp, vp]
    L.meu_slab_fft_inverse_planes.argtypes = [vp, vp, vp, vp]
    L.meu_slab_fft_launch_count.argtypes = [vp]
    L.meu_slab_fft_launch_count.restype = i64
    L.meu_slab_fft_last_error.argtypes = [vp]
    L.meu_slab_fft_last_error.restype = C.c_char_p
    L.meu_slab_fft_destroy.argtypes = [vp]
    L.meu_set_stream.argtypes = [vp, vp]
    L.meu_timing.argtypes = [vp, i32]
    L.meu_timing_report.argtypes = [vp, i32, C.c_char_p, C.POINTER(i64), dp, dp]
    L.meu_timing_report.restype = i32
    L.meu_launch_count.argtypes = [vp]
    L.meu_launch_count.restype = i64
    L.meu_schedule.argtypes = [vp, C.POINTER(i32)]
    L.meu_set_schedule.argtypes = [vp, C.POINTER(i32)]
    L.meu_adjoint.argtypes = [vp, i32, i32, dp, dp, dp, dp, dp]
    L.meu_ensemble_create.argtypes = [i32, C.POINTER(P.MeuParams), i32, C.POINTER(vp)]
    L.meu_ensemble_set_fields.argtypes = [vp, i32, dp, dp]
    L.meu_ensemble_run.argtypes = [vp, i32, C.POINTER(P.MeuDiag)]
    L.meu_ensemble_get_fields.argtypes = [vp, i32, dp, dp, dp]
    L.meu_ensemble_get_step.argtypes = [vp]
    L.meu_ensemble_get_step.restype = i64
    L.meu_ensemble_schedule.argtypes = [vp, i32, C.POINTER(i32)]
    L.meu_ensemble_set_stream.argtypes = [vp, vp]
    L.meu_ensemble_timing.argtypes = [vp, i32]
    L.meu_ensemble_timing_report.argtypes = [vp, i32, C.c_char_p, C.POINTER(i64), dp, dp]
    L.meu_ensemble_timing_report.restype = i32
    L.meu_ensemble_launch_count.argtypes = [vp]
    L.meu_ensemble_launch_count.restype = i64
    L.meu_ensemble_last_error.argtypes = [vp]
    L.meu_ensemble_last_error.restype = C.c_char_p
    L.meu_ensemble_destroy.argtypes = [vp]
    _LIB = L
    return L


def dptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Ran2:
    """The library's host restatement of ran_2 (bit-exact)."""

    def __init__(self, iseed: int):
        self.s = Ran2State()
        lib().meu_ran2_init(C.byref(self.s), int(iseed))

    def __call__(self) -> float:
        return lib().meu_ran2(C.byref(self.s))

    def langevin(self, sd: float) -> float:
        return lib().meu_langevin(C.byref(self.s), float(sd))

    def langevin_fill(self, sd: float, n: int, threads: int = 4) -> np.ndarray:
        """n langevin draws at once (meu_langevin_fill): the numbers of n calls."""
        out = np.empty(n)
        st = lib().meu_langevin_fill(C.byref(self.s), float(sd), int(n), dptr(out), int(threads))
        if st:
            raise MeuError(st, "meu_langevin_fill")
        return out


def init_uniform(nx: int, ny: int, nz: int, nvar: int, seed: int, c0: float, c_amp: float,
                 eta_amp: float) -> Tuple[np.ndarray, np.ndarray]:
    """Uniform-noise initial fields (SoA float64: (1,nz,ny,nx), (nvar,nz,ny,nx))."""
    s = Ran2State()
    lib().meu_ran2_init(C.byref(s), int(seed))
    n3 = nx * ny * nz
    cons = np.empty(n3)
    phi = np.empty(n3 * nvar)
    lib().meu_init_uniform(C.byref(s), nx, ny, nz, nvar, c0, c_amp, eta_amp, dptr(cons), dptr(phi))
    return cons.reshape(1, nz, ny, nx), P.from_fortran(phi, nvar, nx, ny, nz)


def fft_roundtrip(x: np.ndarray, precision: int = P.PREC_F64):
    x = np.ascontiguousarray(x, dtype=np.float64)
    nz, ny, nx = x.shape
    spec = np.empty((nz, ny, nx // 2 + 1), dtype=np.complex128)
    back = np.empty_like(x)
    st = lib().meu_fft_roundtrip(nx, ny, nz, precision, dptr(x), spec.ctypes.data_as(C.POINTER(C.c_double)),
                                 dptr(back))
    if st:
        raise MeuError(st, "meu_fft_roundtrip")
    return spec, back
