"""data_save restart files in the reference's format (CPU: byte layout and
round trip; GPU: a restart continues the run exactly)."""
import os
import struct

import numpy as np
import pytest

from helpers import kks_case
from meumapps_ss_b200 import restart as RS


def test_record_layout_and_round_trip(tmp_path):
    nx, ny, nz, numel, var = 4, 3, 2, 1, 3
    n3 = nx * ny * nz
    rng = np.random.default_rng(1)
    cons, phi, el, u = rng.random(numel * n3), rng.random(var * n3), rng.random(n3), rng.random(12 * n3)
    path = RS.write_data_save(str(tmp_path / "step_0000010"), nx, ny, nz, cons, phi, el, u, numel, var)
    raw = open(path, "rb").read()
    # record 1: 24 bytes of ist/ien framed by markers
    assert struct.unpack("<i", raw[:4])[0] == 24
    assert list(struct.unpack("<6i", raw[4:28])) == [1, 1, 1, nx, ny, nz]
    assert struct.unpack("<i", raw[28:32])[0] == 24
    # record 2: Cons, phi, el_en back to back
    n2 = (numel + var + 1) * n3 * 8
    assert struct.unpack("<i", raw[32:36])[0] == n2
    assert np.array_equal(np.frombuffer(raw[36:36 + numel * n3 * 8], "<f8"), cons)
    assert len(raw) == 32 + (n2 + 8) + 4 * (3 * n3 * 8 + 8)
    d = RS.read_data_save(path, numel, var)
    assert np.array_equal(d["cons"], cons) and np.array_equal(d["phi"], phi)
    assert np.array_equal(d["el_en"], el) and np.array_equal(d["u_state"], u)
    hdr = open(os.path.join(os.path.dirname(path), "data_extract_mult.in")).read().split()
    assert [int(x) for x in hdr] == [nx, ny, nz, 1, var, numel, 1, 1]


def test_corrupt_marker_is_rejected(tmp_path):
    p = tmp_path / "bad"
    p.write_bytes(struct.pack("<i", 8) + b"\0" * 8 + struct.pack("<i", 9))
    with pytest.raises(ValueError):
        RS.read_data_save(str(p), 1, 1)


@pytest.mark.gpu
def test_restart_continues_the_run(tmp_path):
    from meumapps_ss_b200.sim import Simulation
    _, p, cons, phi = kks_case(n=16, nvar=1, steps=20)
    a = Simulation(p)
    a.set_fields(cons, phi)
    a.run(10, diag=False)
    path = RS.save_simulation(a, str(tmp_path / "step_0000010"))
    a.run(10, diag=False)
    b = Simulation(p)
    RS.load_simulation(b, path)
    b.run(10, diag=False)
    ca, fa, _, ua = a.get_fields(ustate=True)
    cb, fb, _, ub = b.get_fields(ustate=True)
    # the displacement state is re-derived from u and its gradients, as in the
    # reference's restart; the elastic fixed point (relative tolerance 1e-7) then
    # converges from a state that differs by round-off
    assert np.max(np.abs(ca - cb)) <= 1e-8 and np.max(np.abs(fa - fb)) <= 1e-8
    assert np.max(np.abs(ua - ub)) <= 1e-6 * max(1.0, np.max(np.abs(ua)))
