"""QRCP selector oracle checks on CPU: the sketch restatement against the
reference's own GaussianRandom + lapack::Orth (compiled in oracle/_ref), and
the basis invariance the GPU selector relies on."""
import numpy as np
import pytest

from oracle import qrcp


def test_sketch_matches_reference_code():
    ref = pytest.importorskip("oracle.ref")
    if not ref.available():
        pytest.skip("oracle/_ref not built on this machine")
    for k1, k2, p, seed in [(16, 12, 9, 41), (32, 32, 22, 2), (7, 9, 5, 123)]:
        g1, g2 = ref.qrcp_sketch(k1, k2, p, seed, orth=False)
        r1, r2 = qrcp.gaussians(k1, k2, p, seed)
        assert np.array_equal(g1, r1) and np.array_equal(g2, r2)
        g1, g2 = ref.qrcp_sketch(k1, k2, p, seed, orth=True)
        o1, o2 = qrcp.sketch(k1, k2, p, seed)
        assert np.array_equal(g1, o1) and np.array_equal(g2, o2)


def test_iround_and_num_pre():
    assert qrcp.num_pre(2048, 1.5) == 55
    assert qrcp.num_pre(2048, 2.5) == 72
    assert qrcp.num_pre(4320, 2.5) == 104
    assert qrcp.iround(2.5) == 3 and qrcp.iround(-2.5) == -3


def test_pivots_depend_only_on_the_sketch_span():
    """An orthogonal change of basis of G1, G2 leaves the CPQR pivots alone."""
    rng = np.random.default_rng(3)
    psi = np.linalg.qr(rng.standard_normal((900, 10)))[0]
    g1, g2 = qrcp.sketch(10, 10, 6, 41)
    h1 = np.linalg.qr(qrcp.gaussians(10, 10, 6, 41)[0])[0]
    h2 = np.linalg.qr(qrcp.gaussians(10, 10, 6, 41)[1])[0]
    a = qrcp.select(psi, 5, 5, 5, 5, 5, 24, g=(g1, g2))
    b = qrcp.select(psi, 5, 5, 5, 5, 5, 24, g=(h1, h2))
    assert a[1] == b[1]
    assert np.array_equal(a[2][:24], b[2][:24])
