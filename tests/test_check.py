"""Pins the numpy check restatement (oracle/check.py) against the numbers the
reference's own checkcode printed (goldens)."""
import pytest

from conftest import load_golden
from oracle import check


@pytest.mark.parametrize("name", ["small_s1s2", "small_mu0"])
def test_check_restatement_matches_reference(name):
    g = load_golden(name)
    a = (int(g["nocc"]), int(g["nv1"]), int(g["nc1"]), int(g["nv2"]), int(g["nc2"]))
    fe, ce = check.check(g["psi"], tuple(int(x) for x in g["ng"]), tuple(g["length"]), *a,
                         int(g["rk_eff"]), g["piv"], g["theta"])
    assert abs(fe / float(g["fit_err"]) - 1) < 1e-12
    assert abs(ce / float(g["coul_err"]) - 1) < 1e-6
