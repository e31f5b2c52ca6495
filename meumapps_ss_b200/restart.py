"""Restart and post-processing files in the reference's own format.

The reference writes, every `ifreq` steps, a directory `step_NNNNNNN` holding
* `data_extract_mult.in`: list-directed `Nx Ny Nz nprocs vartot numel` and the
  process grid `dims` (Multi_MEUMAPPS.f:1078-1083), read by data_ext_modular.f;
* `data_save.NNNN` (one per MPI rank, NNNN = rank + 1): a Fortran unformatted
  sequential file of six records (Multi_MEUMAPPS.f:1087-1094): `ist, ien`
  (integer*4 x 3 each), then `Cons, phi, el_en`, then `u1, u2, u3`, then the
  gradients `grad_j_u1..u3` for j = 1, 2, 3 (real*8, Fortran order, the
  component index of Cons and phi fastest).  The restart path reads the same
  records back (Multi_MEUMAPPS.f:470-481).
A GPU run is one rank: dims = (1, 1), ist = (1, 1, 1), ien = (Nx, Ny, Nz).

Unformatted sequential records are framed by 4-byte little-endian length
markers before and after the payload, as gfortran and most Unix compilers
write them.  Records of 2 GiB or more would need the compiler-specific
subrecord scheme and are rejected.
"""
from __future__ import annotations

import os
import struct
from typing import Dict, Optional

import numpy as np

_MAX_RECORD = 2 ** 31 - 9


def _write_record(f, *arrays) -> None:
    payload = b"".join(np.ascontiguousarray(a).tobytes() for a in arrays)
    if len(payload) > _MAX_RECORD:
        raise ValueError(f"record of {len(payload)} bytes exceeds the 2 GiB sequential-record limit")
    mark = struct.pack("<i", len(payload))
    f.write(mark)
    f.write(payload)
    f.write(mark)


def _read_record(f) -> bytes:
    head = f.read(4)
    if len(head) != 4:
        raise EOFError("truncated record marker")
    (n,) = struct.unpack("<i", head)
    if n < 0:
        raise ValueError("subrecords (records of 2 GiB or more) are not supported")
    data = f.read(n)
    (tail,) = struct.unpack("<i", f.read(4))
    if tail != n or len(data) != n:
        raise ValueError("corrupt record markers")
    return data


def write_data_save(directory: str, nx: int, ny: int, nz: int, cons_f: np.ndarray, phi_f: np.ndarray,
                    el_en: np.ndarray, u_state: Optional[np.ndarray], numel: int, vartot: int) -> str:
    """Write `directory/data_save.0001` and `directory/data_extract_mult.in`.

    cons_f, phi_f: Fortran-layout flat arrays (component fastest, as meu_get_fields
    returns them); el_en: Nx*Ny*Nz; u_state: the 12 fields in data_save order
    (u1..u3, grad_1_u1..u3, grad_2_u1..u3, grad_3_u1..u3), or None for zeros
    (decks without a displacement state)."""
    n3 = nx * ny * nz
    cons_f = np.asarray(cons_f, dtype="<f8").reshape(-1)
    phi_f = np.asarray(phi_f, dtype="<f8").reshape(-1)
    el_en = np.asarray(el_en, dtype="<f8").reshape(-1)
    if cons_f.size != numel * n3 or phi_f.size != vartot * n3 or el_en.size != n3:
        raise ValueError("field sizes do not match the grid")
    u = np.zeros(12 * n3, dtype="<f8") if u_state is None else np.asarray(u_state, dtype="<f8").reshape(-1)
    if u.size != 12 * n3:
        raise ValueError("u_state must hold 12 fields")
    os.makedirs(directory, exist_ok=True)
    with open(os.path.join(directory, "data_extract_mult.in"), "w") as f:
        f.write(f" {nx:11d} {ny:11d} {nz:11d} {1:11d} {vartot:11d} {numel:11d}\n")
        f.write(f" {1:11d} {1:11d}\n")
    path = os.path.join(directory, "data_save.0001")
    with open(path, "wb") as f:
        _write_record(f, np.array([1, 1, 1, nx, ny, nz], dtype="<i4"))
        _write_record(f, cons_f, phi_f, el_en)
        _write_record(f, u[:3 * n3])
        for j in range(3):
            _write_record(f, u[(3 + 3 * j) * n3:(6 + 3 * j) * n3])
    return path


def read_data_save(path: str, numel: int, vartot: int) -> Dict[str, np.ndarray]:
    """Read a one-rank data_save file: dict with ist, ien, cons, phi (Fortran
    layout, flat), el_en and u_state (12 fields, flat)."""
    with open(path, "rb") as f:
        idx = np.frombuffer(_read_record(f), dtype="<i4")
        ist, ien = idx[:3].copy(), idx[3:6].copy()
        n3 = int(np.prod(ien - ist + 1))
        rec = np.frombuffer(_read_record(f), dtype="<f8")
        if rec.size != (numel + vartot + 1) * n3:
            raise ValueError("field record does not match numel, vartot and the grid")
        cons = rec[:numel * n3].copy()
        phi = rec[numel * n3:(numel + vartot) * n3].copy()
        el = rec[(numel + vartot) * n3:].copy()
        u = np.concatenate([np.frombuffer(_read_record(f), dtype="<f8") for _ in range(4)])
    return {"ist": ist, "ien": ien, "cons": cons, "phi": phi, "el_en": el, "u_state": u}


def save_simulation(sim, directory: str, ustate: bool = True) -> str:
    """meu_get_fields of a Simulation into the reference's restart files."""
    p = sim.params
    n3 = p.nx * p.ny * p.nz
    cons = np.empty(p.numel * n3)
    phi = np.empty(p.nvar * n3)
    el = np.empty(n3)
    u = np.empty(12 * n3) if ustate else None
    sim.get_fields_fortran(cons, phi, el, u)
    return write_data_save(directory, p.nx, p.ny, p.nz, cons, phi, el, u, p.numel, p.nvar)


def load_simulation(sim, path: str, ustate: bool = True) -> None:
    """meu_set_fields of a Simulation from a data_save file (the reference's restart)."""
    p = sim.params
    d = read_data_save(path, p.numel, p.nvar)
    sim.set_fields_fortran(d["cons"], d["phi"], d["u_state"] if ustate else None)
