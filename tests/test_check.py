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


@pytest.mark.parametrize("name", ["small_s1s2", "small_mu0"])
def test_sampled_check_restatement(name):
    """The sampled check: with every pair listed it is the full check; on a
    subset, the fitted-density spectra give the reference's c^T A c form."""
    import numpy as np

    g = load_golden(name)
    a = (int(g["nocc"]), int(g["nv1"]), int(g["nc1"]), int(g["nv2"]), int(g["nc2"]))
    ng, ln = tuple(int(x) for x in g["ng"]), tuple(g["length"])
    rk = int(g["rk_eff"])
    npair = (a[1] + a[2]) * (a[3] + a[4])
    full = check.check(g["psi"], ng, ln, *a, rk, g["piv"], g["theta"])
    every = check.check_sampled(g["psi"], ng, ln, *a, rk, g["piv"], g["theta"], np.arange(npair))
    # relative errors near 1e-9 (small_mu0 fits almost exactly) are differences of
    # nearly equal sums: compared to 1e-8 of the value plus 1e-15 absolute
    close = lambda x, y: abs(x - y) <= 1e-8 * abs(y) + 1e-15  # noqa: E731
    assert close(every[0], full[0]) and close(every[1], full[1])
    sub = np.random.default_rng(0).choice(npair, size=npair // 3, replace=False)
    ref_form = check.check_sampled(g["psi"], ng, ln, *a, rk, g["piv"], g["theta"], sub)
    fd_form = check.check_sampled(g["psi"], ng, ln, *a, rk, g["piv"], g["theta"], sub,
                                  fitted_spectra=True)
    assert close(fd_form[0], ref_form[0]) and close(fd_form[1], ref_form[1])
