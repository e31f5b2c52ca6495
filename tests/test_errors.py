"""The reference's stops, made on the host: each error deck drives the CPU oracle
to the status code the reference's err_flag carries (the GPU tests in
test_gpu_errors.py check the library against the same decks), and the host
set-up stops with code 20 on a singular stiffness (ModInitials.f:98)."""
import pytest

import helpers as H
from meumapps_ss_b200 import configs as CF
from meumapps_ss_b200 import params as P

DECKS = [H.singular_q_deck, H.singular_mix_deck, H.singular_elener_deck, H.singular_z_deck,
         H.diverging_elastic_deck]


@pytest.mark.parametrize("deck", DECKS, ids=lambda f: f.__name__)
def test_oracle_stops_with_the_reference_code(oracle, deck):
    p, c, e, code = deck()
    o = oracle.OracleSim(p)
    o.set_fields(c, e)
    with pytest.raises(RuntimeError, match=f"status {code}$"):
        o.run(3)


def test_setup_stops_on_singular_stiffness():
    txt = CF.kks_input_txt(16, 1, 5)
    # the precipitate's C44 = 0: InitElasticMat's invert(C, 6) fails its rcond test
    txt = txt.replace("1.80e11 1.00e11 0.50e11", "1.80e11 1.00e11 0.0")
    with pytest.raises(P.SetupError) as ex:
        P.kks_params(P.parse_input_txt(txt))
    assert ex.value.code == 20
