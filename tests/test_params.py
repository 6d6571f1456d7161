"""The .nml reader and initial states mirror the reference
(parametres.c, hydro_funcs.c); expected values come from the reference's own
reader (tests/golden/nml_parse.json) and the oracle's init."""
import glob
import json
import os

import numpy as np
import pytest

from hydro_b200 import init_state, make_params, read_nml
from _helpers import bitwise_equal, orc_from_H

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "nml", "*.nml"))))
def test_nml_reader_matches_reference(path):
    want = json.load(open(os.path.join(GOLDEN, "nml_parse.json")))[os.path.basename(path)]
    H = read_nml(path)
    for k, v in want.items():
        assert getattr(H, k) == v, k


def test_unknown_scheme_is_rejected(tmp_path):
    p = tmp_path / "bad.nml"
    p.write_text("scheme=godunov\n")
    with pytest.raises(ValueError):
        read_nml(str(p))


@pytest.mark.parametrize("tc", [0, 1, 2])
@pytest.mark.parametrize("nx,ny", [(250, 125), (33, 18), (4, 7)])
def test_init_matches_oracle(oracle, tc, nx, ny):
    H = make_params(nx, ny, testcase=tc)
    u = init_state(H)
    o = oracle.init_state(orc_from_H(oracle, H), tc)
    assert bitwise_equal(u, o)


def test_corner_case_dx_is_one_over_nx():
    H = read_nml(os.path.join(GOLDEN, "nml", "corner_250x125.nml"))
    assert H.dx == 1.0 / 250
    assert (H.nxt, H.nyt, H.nxyt) == (254, 129, 254)
