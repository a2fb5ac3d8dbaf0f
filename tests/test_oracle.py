"""Pins the oracle: the CPU restatements (oracle/kmeans_port.cpp, oracle/fit.py)
against the golden fixtures that the reference's own CPU code produced
(tests/golden/make_golden.py), and against that code itself when it is built
here (oracle/_ref)."""
import numpy as np
import pytest

from conftest import load_golden
from oracle import fit as ofit
from oracle import port

CASES = ["si8_example", "small_s1s2", "small_mu0", "small_iters0", "small_early"]


def _args(g):
    return (tuple(int(x) for x in g["ng"]), tuple(float(x) for x in g["length"]), int(g["nocc"]),
            int(g["nv1"]), int(g["nc1"]), int(g["nv2"]), int(g["nc2"]))


@pytest.mark.parametrize("name", CASES)
def test_port_kmeans_matches_reference_golden(name):
    g = load_golden(name)
    ng, length, nocc, nv1, nc1, nv2, nc2 = _args(g)
    piv, rk, it, w = port.kmeans_piv(g["psi"], ng, length, nocc, nv1, nc1, nv2, nc2,
                                     int(g["rk_requested"]), int(g["iters"]),
                                     rand_seed=int(g["rand_seed"]))
    assert np.array_equal(w, g["weight"])  # bit-exact weight
    assert rk == int(g["rk_eff"]) and it == int(g["n_iter"])
    assert np.array_equal(piv, g["piv"])  # bit-exact pivots


@pytest.mark.parametrize("name", ["small_s1s2", "small_mu0", "small_iters0"])
def test_fit_restatement_matches_reference_golden(name):
    g = load_golden(name)
    ng, length, nocc, nv1, nc1, nv2, nc2 = _args(g)
    rk = int(g["rk_eff"])
    th = ofit.getbasis(g["psi"], nocc, nv1, nc1, nv2, nc2, rk, g["piv"])
    ref_th = g["theta"]
    # fitted pair densities are well conditioned; theta carries cond(C C^T) * eps
    fd = ofit.fitted_densities(th, g["psi"], nocc, nv1, nc1, nv2, nc2, rk, g["piv"])
    fd_ref = ofit.fitted_densities(ref_th, g["psi"], nocc, nv1, nc1, nv2, nc2, rk, g["piv"])
    assert ofit.rel(fd, fd_ref) < 1e-8
    assert ofit.rel(th, ref_th) < 1e-5


def test_port_and_reference_agree_live():
    ref = pytest.importorskip("oracle.ref")
    if not ref.available():
        pytest.skip("oracle/_ref not built on this machine")
    g = load_golden("small_s1s2")
    rng = np.random.default_rng(5)
    psi = np.asfortranarray(np.linalg.qr(rng.standard_normal((8 * 9 * 10, 7)))[0])
    for mu, iters in [(20, 0), (20, 3), (33, 40)]:
        a = ref.kmeans_piv(psi, (8, 9, 10), (7.0, 8.0, 9.5), 3, 3, 4, 2, 1, mu, iters,
                           cross_check=True)
        b = port.kmeans_piv(psi, (8, 9, 10), (7.0, 8.0, 9.5), 3, 3, 4, 2, 1, mu, iters)
        assert a[1:3] == b[1:3]
        assert np.array_equal(a[0], b[0])
    assert g["piv"].dtype == np.int32


@pytest.mark.parametrize("seed", range(8))
def test_port_and_reference_agree_on_random_shapes(seed):
    """Random odd and even grids, state windows (S1 != S2 included), mu and
    iteration caps: the port's weights and pivots equal the reference code's
    bit for bit."""
    ref = pytest.importorskip("oracle.ref")
    if not ref.available():
        pytest.skip("oracle/_ref not built on this machine")
    rng = np.random.default_rng(100 + seed)
    ng = tuple(int(x) for x in rng.integers(5, 13, size=3))
    n = ng[0] * ng[1] * ng[2]
    nstate = int(rng.integers(4, 10))
    nocc = int(rng.integers(2, nstate - 1))
    nv1, nv2 = int(rng.integers(1, nocc + 1)), int(rng.integers(1, nocc + 1))
    nc1, nc2 = int(rng.integers(0, nstate - nocc + 1)), int(rng.integers(0, nstate - nocc + 1))
    length = tuple(float(x) for x in rng.uniform(5.0, 12.0, size=3))
    mu = int(rng.integers(4, min(64, n // 4)))
    iters = int(rng.choice([0, 1, 5, 30]))
    psi = np.asfortranarray(np.linalg.qr(rng.standard_normal((n, nstate)))[0])
    w_ref = ref.weight(psi, nocc, nv1, nc1, nv2, nc2)
    a = ref.kmeans_piv(psi, ng, length, nocc, nv1, nc1, nv2, nc2, mu, iters)
    b = port.kmeans_piv(psi, ng, length, nocc, nv1, nc1, nv2, nc2, mu, iters)
    assert np.array_equal(b[3], w_ref)
    assert a[1:3] == b[1:3]
    assert np.array_equal(a[0], b[0])


@pytest.mark.parametrize("seed", range(4))
def test_fit_restatement_and_reference_agree_on_random_shapes(seed):
    """The numpy fit (oracle/fit.py) against the reference's getbasis on random
    shapes, with pivots from the reference's own K-means: fitted pair densities
    to 1e-8 (theta itself carries cond(C C^T) x eps)."""
    ref = pytest.importorskip("oracle.ref")
    if not ref.available():
        pytest.skip("oracle/_ref not built on this machine")
    rng = np.random.default_rng(200 + seed)
    ng = tuple(int(x) for x in rng.integers(6, 12, size=3))
    n = ng[0] * ng[1] * ng[2]
    nstate = int(rng.integers(5, 10))
    nocc = int(rng.integers(2, nstate - 1))
    nv1, nv2 = int(rng.integers(1, nocc + 1)), int(rng.integers(1, nocc + 1))
    nc1, nc2 = int(rng.integers(1, nstate - nocc + 1)), int(rng.integers(1, nstate - nocc + 1))
    length = tuple(float(x) for x in rng.uniform(5.0, 12.0, size=3))
    mu = int(rng.integers(8, min(48, (nv1 + nc1) * (nv2 + nc2) + 1)))
    psi = np.asfortranarray(np.linalg.qr(rng.standard_normal((n, nstate)))[0])
    piv, rk, _, _ = ref.kmeans_piv(psi, ng, length, nocc, nv1, nc1, nv2, nc2, mu, 10)
    a = (nocc, nv1, nc1, nv2, nc2)
    th_ref = ref.getbasis(psi, ng, length, *a, rk, piv)
    th = ofit.getbasis(psi, *a, rk, piv)
    fd = ofit.fitted_densities(th, psi, *a, rk, piv)
    fd_ref = ofit.fitted_densities(th_ref, psi, *a, rk, piv)
    assert ofit.rel(fd, fd_ref) < 1e-8


def test_sampled_row_fit_equals_full_fit_rows():
    """oracle.fit.getbasis_rows (the fit evaluated on sampled grid rows, used
    at the full benchmark sizes) gives exactly the rows of the full fit."""
    rng = np.random.default_rng(0)
    psi = np.linalg.qr(rng.standard_normal((3000, 10)))[0]
    piv = rng.choice(3000, size=40, replace=False).astype(np.int32)
    rows = np.sort(rng.choice(3000, size=100, replace=False))
    for a in [(5, 5, 5, 5, 5), (5, 5, 3, 2, 4)]:
        full = ofit.getbasis(psi, *a, 40, piv)
        assert np.array_equal(full[rows], ofit.getbasis_rows(psi, *a, 40, piv, rows))


@pytest.mark.parametrize("name", CASES[:4])
def test_port_warm_start_matches_reference_live(name):
    """The port's K-means warm start (previous pivots as initial centroids,
    utility.cpp:725-749) against the reference's own KMEAN given the same
    previous piv."""
    ref = pytest.importorskip("oracle.ref")
    if not ref.available():
        pytest.skip("oracle/_ref not built on this machine")
    g = load_golden(name)
    ng, length = tuple(int(x) for x in g["ng"]), tuple(float(x) for x in g["length"])
    mu, iters = int(g["rk_requested"]), int(g["iters"])
    rng = np.random.default_rng(1)
    w2 = np.abs(g["weight"] * (1 + 0.05 * rng.standard_normal(g["weight"].shape)))
    prev, _, _ = port.kmeans(w2, ng, length, mu, iters)
    a = port.kmeans_warm(g["weight"], ng, length, mu, iters, prev)
    b = ref.kmeans_warm(g["weight"], ng, length, mu, iters, prev)
    assert np.array_equal(a[0], b[0]) and a[1:] == b[1:]
    assert a[3] > 0  # previous pivots were reused
