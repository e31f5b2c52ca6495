"""Python mirror of the reference's time-loop interface over the C-ABI.

``Simulation`` is what the Fortran driver does around its ``goto 4`` loop
(Multi_MEUMAPPS.f:548-1106): hand the fields over, advance ``nsteps`` time
steps, read the per-step fort.98 / fort.99 diagnostics and the fields back for
the data_save writer.  Arrays are structure-of-arrays ``(ncomp, nz, ny, nx)``
float64 here; the C-ABI itself takes the reference's Fortran layout
(component index fastest), which ``set_fields_fortran`` passes through as is.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Optional, Tuple

import numpy as np

from . import params as P
from ._lib import MeuError, dptr, lib


class Simulation:
    def __init__(self, params: P.MeuParams):
        self.params = params.copy()
        h = C.c_void_p()
        st = lib().meu_create(C.byref(self.params), C.byref(h))
        if st:
            raise MeuError(st, lib().meu_last_error(None).decode())
        self.h = h
        p = self.params
        self.shape = (p.nz, p.ny, p.nx)

    # -- life cycle --
    def close(self) -> None:
        if getattr(self, "h", None):
            lib().meu_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int) -> None:
        if st:
            raise MeuError(st, lib().meu_last_error(self.h).decode())

    # -- fields --
    def set_fields(self, cons: np.ndarray, phi: np.ndarray, ustate: Optional[np.ndarray] = None) -> None:
        c = P.to_fortran(cons)
        f = P.to_fortran(phi)
        u = None if ustate is None else np.ascontiguousarray(ustate, dtype=np.float64).reshape(-1)
        self.set_fields_fortran(c, f, u)

    def set_fields_fortran(self, cons: Optional[np.ndarray], phi: Optional[np.ndarray],
                           ustate: Optional[np.ndarray] = None) -> None:
        self._check(lib().meu_set_fields(self.h, dptr(cons), dptr(phi), dptr(ustate)))

    def add_noise(self, incr: np.ndarray) -> None:
        self._check(lib().meu_add_noise(self.h, dptr(P.to_fortran(incr))))

    def get_fields(self, ustate: bool = False) -> Tuple[np.ndarray, np.ndarray, np.ndarray, Optional[np.ndarray]]:
        p = self.params
        n3 = p.nx * p.ny * p.nz
        cons = np.empty(p.numel * n3)
        phi = np.empty(p.nvar * n3)
        el = np.empty(n3)
        u = np.empty(12 * n3) if ustate else None
        self._check(lib().meu_get_fields(self.h, dptr(cons), dptr(phi), dptr(el), dptr(u)))
        nx, ny, nz = p.nx, p.ny, p.nz
        return (P.from_fortran(cons, p.numel, nx, ny, nz), P.from_fortran(phi, p.nvar, nx, ny, nz),
                el.reshape(nz, ny, nx), None if u is None else u.reshape(12, nz, ny, nx))

    def get_fields_fortran(self, cons: Optional[np.ndarray], phi: Optional[np.ndarray],
                           el: Optional[np.ndarray] = None, ustate: Optional[np.ndarray] = None) -> None:
        self._check(lib().meu_get_fields(self.h, dptr(cons), dptr(phi), dptr(el), dptr(ustate)))

    # -- time loop --
    def run(self, nsteps: int, diag: bool = True) -> Optional[Dict[str, np.ndarray]]:
        rows = (P.MeuDiag * max(int(nsteps), 1))() if diag else None
        self._check(lib().meu_run(self.h, int(nsteps), rows))
        if not diag:
            return None
        return P.diag_to_dict(list(rows)[:nsteps])

    # -- instrumentation --
    def set_stream(self, stream_ptr: int) -> None:
        self._check(lib().meu_set_stream(self.h, C.c_void_p(int(stream_ptr)) if stream_ptr else None))

    def timing(self, enable: bool) -> None:
        self._check(lib().meu_timing(self.h, 1 if enable else 0))

    def timing_report(self) -> Dict[str, Dict[str, float]]:
        mx = 64
        names = C.create_string_buffer(32 * mx)
        cnt = (C.c_int64 * mx)()
        ms = (C.c_double * mx)()
        by = (C.c_double * mx)()
        n = lib().meu_timing_report(self.h, mx, names, cnt, ms, by)
        if n < 0:
            raise MeuError(-n, lib().meu_last_error(self.h).decode())
        out = {}
        for i in range(min(n, mx)):
            nm = names.raw[32 * i:32 * i + 32].split(b"\0")[0].decode()
            out[nm] = {"launches": int(cnt[i]), "ms": float(ms[i]), "bytes": float(by[i])}
        return out

    @property
    def launch_count(self) -> int:
        return int(lib().meu_launch_count(self.h))

    @property
    def step(self) -> int:
        return int(lib().meu_get_step(self.h))
