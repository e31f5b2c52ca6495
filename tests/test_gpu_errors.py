"""The library's status codes for the reference's stops, on the GPU, from
inputs made on the host (no fault is provoked): singular Omega(k) (3), singular
compliance mixes in eldis (4) and elener (6), singular interface-composition
solve (2), elastic divergence (7, the call returns), and non-finite fields
(104).  After each error the handle (or a fresh one) runs a good deck."""
import time

import numpy as np
import pytest

import helpers as H
from meumapps_ss_b200 import params as P
from meumapps_ss_b200._lib import MeuError
from meumapps_ss_b200.sim import Simulation


def _expect(p, c, e, code, steps=3):
    t0 = time.time()
    with Simulation(p) as g:
        g.set_fields(c, e)
        with pytest.raises(MeuError) as ex:
            g.run(steps)
        assert ex.value.code == code, str(ex.value)
    assert time.time() - t0 < 120
    # the context is still usable: a good deck runs on a new handle
    q, c2, e2 = H.active_landau(16, 1)
    with Simulation(q) as g:
        g.set_fields(c2, e2)
        g.run(2)


@pytest.mark.gpu
@pytest.mark.parametrize("generic", [False, True])
def test_singular_q(generic):
    p, c, e, code = H.singular_q_deck()
    if generic:
        p.flags |= P.FLAG_GENERIC
    _expect(p, c, e, code)


@pytest.mark.gpu
@pytest.mark.parametrize("deck", [H.singular_mix_deck, H.singular_elener_deck, H.singular_z_deck,
                                  H.diverging_elastic_deck], ids=lambda f: f.__name__)
def test_reference_stops(deck):
    p, c, e, code = deck()
    _expect(p, c, e, code)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["fused", "generic", "kks"])
def test_non_finite_fields(case):
    if case == "kks":
        _, p, c, e = H.kks_case(16, 1, 5)
    else:
        p, c, e = H.active_landau(16, 2)
        if case == "generic":
            p.flags |= P.FLAG_GENERIC
    bad = c.copy()
    bad[0, 3, 4, 5] = np.nan
    with Simulation(p) as g:
        g.set_fields(bad, e)
        with pytest.raises(MeuError) as ex:
            g.run(4)
        assert ex.value.code == 104, str(ex.value)
        # the same handle takes good fields and runs on
        g.set_fields(c, e)
        d = g.run(4)
        assert np.all(np.isfinite(d["etot"]))
