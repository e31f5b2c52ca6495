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

    def run_into(self, nsteps: int, rows) -> None:
        """meu_run into a caller-allocated ``(P.MeuDiag * nsteps)()`` buffer, with no
        conversion afterwards: exactly the call a Fortran or C driver makes (for timing)."""
        self._check(lib().meu_run(self.h, int(nsteps), rows))

    def run_noise(self, nsteps: int, rng, sd: float, diag: bool = True) -> Optional[Dict[str, np.ndarray]]:
        """meu_run_noise: the steps with step <= noise_step draw their Langevin increments
        from ``rng`` (a ``_lib.Ran2State``, advanced in place) on a host thread."""
        rows = (P.MeuDiag * max(int(nsteps), 1))() if diag else None
        self._check(lib().meu_run_noise(self.h, int(nsteps), C.byref(rng), float(sd), rows))
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

    @property
    def schedule(self) -> Optional[Tuple[int, int, int]]:
        """(radix plan variant, plane threads, column tile) of the fused step; on the
        generic path (radix plan of the power-of-two transforms, 0, column-tile factor)."""
        out = (C.c_int32 * 3)()
        if lib().meu_schedule(self.h, out):
            return None
        return tuple(int(x) for x in out)

    def adjoint(self, nsteps: int, checkpoint_every: int, c_target: np.ndarray, eta_target: np.ndarray,
                want_field: bool = True):
        """Loss J = 1/(2 N^3) sum [(eta_T - eta*)^2 + (c_T - c*)^2] after nsteps steps from the
        current fields and its gradient (meu_adjoint).  Returns (J, dict, dJ/deta_0 or None);
        the dict holds dJ/d of beta (kappa_eta scale), kappa_c, L, M and alpha (eigenstrain scale)."""
        p = self.params
        ct = P.to_fortran(c_target)
        et = P.to_fortran(eta_target)
        loss = C.c_double()
        dpar = (C.c_double * 5)()
        g = np.empty(p.nvar * p.nx * p.ny * p.nz) if want_field else None
        self._check(lib().meu_adjoint(self.h, int(nsteps), int(checkpoint_every), dptr(ct), dptr(et),
                                      C.byref(loss), dpar, dptr(g)))
        names = ("beta_eta", "kappa_c", "L", "M", "alpha")
        grads = {k: float(v) for k, v in zip(names, dpar)}
        if g is None:
            field = None
        elif p.nvar == 1:
            field = g.reshape(p.nz, p.ny, p.nx)
        else:  # (nvar, nz, ny, nx) from the phi(vartot,Nx,Ny,Nz) layout
            field = P.from_fortran(g, p.nvar, p.nx, p.ny, p.nz)
        return float(loss.value), grads, field

    def set_schedule(self, pv: int, ntp: int, tm: int) -> None:
        """Pick the fused step's schedule (before the first set_fields), or the generic
        path's transform plan as (0 or 2, 0, 1 or 2)."""
        self._check(lib().meu_set_schedule(self.h, (C.c_int32 * 3)(pv, ntp, tm)))


def schedule_candidates(n: int, f64: bool):
    """Schedules of the fused step instantiated for an n^3 grid (the autotuner's candidates)."""
    wide = 8 if f64 else 16
    cols = n * (n // 2 + 1)
    return [(pv, ntp, tm) for pv in (0, 1, 2) for ntp in (512, 256) for tm in (wide, wide // 2)
            if cols % tm == 0 and cols // tm <= 2048]


def _timing_table(fn, h) -> Dict[str, Dict[str, float]]:
    mx = 64
    names = C.create_string_buffer(32 * mx)
    cnt = (C.c_int64 * mx)()
    ms = (C.c_double * mx)()
    by = (C.c_double * mx)()
    n = fn(h, mx, names, cnt, ms, by)
    if n < 0:
        raise MeuError(-n, "timing report failed")
    out = {}
    for i in range(min(n, mx)):
        nm = names.raw[32 * i:32 * i + 32].split(b"\0")[0].decode()
        out[nm] = {"launches": int(cnt[i]), "ms": float(ms[i]), "bytes": float(by[i])}
    return out


class Ensemble:
    """Many independent fused Landau simulations advanced together
    (``meu_ensemble_*``).  ``params`` is a list of decks; member m's fields are
    set and read as for ``Simulation``.  ``autotune`` times the schedule variants
    of every size bucket at creation.  ``persistent`` runs the warm steps of every
    member as work items of one persistent launch (``MEU_ENS_PERSISTENT``: one order
    parameter per member, schedule (2, 256, wide tile) for every size)."""

    def __init__(self, params, autotune: bool = False, persistent: bool = False):
        self.params = [p.copy() for p in params]
        arr = (P.MeuParams * len(self.params))(*self.params)
        h = C.c_void_p()
        flags = (1 if autotune else 0) | (2 if persistent else 0)
        st = lib().meu_ensemble_create(len(self.params), arr, flags, C.byref(h))
        if st:
            raise MeuError(st, lib().meu_ensemble_last_error(None).decode())
        self.h = h

    def __len__(self) -> int:
        return len(self.params)

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().meu_ensemble_destroy(self.h)
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
            raise MeuError(st, lib().meu_ensemble_last_error(self.h).decode())

    def set_fields(self, m: int, cons: np.ndarray, phi: np.ndarray) -> None:
        self.set_fields_fortran(m, P.to_fortran(cons), P.to_fortran(phi))

    def set_fields_fortran(self, m: int, cons: Optional[np.ndarray], phi: Optional[np.ndarray]) -> None:
        self._check(lib().meu_ensemble_set_fields(self.h, int(m), dptr(cons), dptr(phi)))

    def get_fields(self, m: int) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        p = self.params[m]
        n3 = p.nx * p.ny * p.nz
        cons = np.empty(p.numel * n3)
        phi = np.empty(p.nvar * n3)
        el = np.empty(n3)
        self._check(lib().meu_ensemble_get_fields(self.h, int(m), dptr(cons), dptr(phi), dptr(el)))
        nx, ny, nz = p.nx, p.ny, p.nz
        return P.from_fortran(cons, p.numel, nx, ny, nz), P.from_fortran(phi, p.nvar, nx, ny, nz), el.reshape(nz, ny, nx)

    def get_fields_fortran(self, m: int, cons: Optional[np.ndarray], phi: Optional[np.ndarray],
                           el: Optional[np.ndarray] = None) -> None:
        self._check(lib().meu_ensemble_get_fields(self.h, int(m), dptr(cons), dptr(phi), dptr(el)))

    def run_into(self, nsteps: int, rows) -> None:
        """meu_ensemble_run into a caller-allocated ``(P.MeuDiag * (members * nsteps))()``
        buffer, with no conversion afterwards (for timing)."""
        self._check(lib().meu_ensemble_run(self.h, int(nsteps), rows))

    def run(self, nsteps: int, diag: bool = True):
        """Advance every member; returns one diagnostics dict per member (or None)."""
        n = len(self.params)
        rows = (P.MeuDiag * max(int(nsteps) * n, 1))() if diag else None
        self._check(lib().meu_ensemble_run(self.h, int(nsteps), rows))
        if not diag:
            return None
        lst = list(rows)
        return [P.diag_to_dict(lst[m * nsteps:(m + 1) * nsteps]) for m in range(n)]

    def schedule(self, m: int) -> Tuple[int, int, int, int]:
        """(radix plan variant, plane threads, column tile, bucket) of member m."""
        out = (C.c_int32 * 4)()
        self._check(lib().meu_ensemble_schedule(self.h, int(m), out))
        return tuple(int(x) for x in out)

    def set_stream(self, stream_ptr: int) -> None:
        self._check(lib().meu_ensemble_set_stream(self.h, C.c_void_p(int(stream_ptr)) if stream_ptr else None))

    def timing(self, enable: bool) -> None:
        self._check(lib().meu_ensemble_timing(self.h, 1 if enable else 0))

    def timing_report(self) -> Dict[str, Dict[str, float]]:
        return _timing_table(lib().meu_ensemble_timing_report, self.h)

    @property
    def launch_count(self) -> int:
        return int(lib().meu_ensemble_launch_count(self.h))

    @property
    def step(self) -> int:
        return int(lib().meu_ensemble_get_step(self.h))
