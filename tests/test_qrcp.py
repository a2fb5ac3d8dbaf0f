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


def _cancellation_matrix(seed):
    """Columns nearly parallel to the first pivot: after one step their
    residual norms are ~1e-6 of the originals, where downdating loses about
    4 digits and dgeqpf recomputes (LAPACK Working Note 176)."""
    rng = np.random.default_rng(seed)
    m, n = 40, 60
    v1 = rng.standard_normal(m)
    v1 /= np.linalg.norm(v1) * 0.5
    a = np.zeros((m, n))
    a[:, 0] = v1 * 10
    for j in range(1, n):
        w = rng.standard_normal(m)
        w -= v1 * (v1 @ w) / (v1 @ v1)
        w /= np.linalg.norm(w)
        a[:, j] = v1 * (1.0 + 1e-9 * j) + (1e-6 * (1 + 1e-6 * rng.standard_normal())) * w
    return np.asfortranarray(a)


def test_dgeqpf_port_matches_lapack():
    """oracle/qrcp_port.cpp (port_dgeqpf) takes LAPACK dgeqpf's pivots,
    including where only a recomputed norm orders the columns correctly."""
    rng = np.random.default_rng(0)
    u = np.linalg.qr(rng.standard_normal((100, 100)))[0]
    v = np.linalg.qr(rng.standard_normal((300, 100)))[0]
    cases = [rng.standard_normal((30, 50)), rng.standard_normal((80, 40)),
             _cancellation_matrix(0), _cancellation_matrix(1),
             u @ np.diag(np.logspace(0, -14, 100)) @ v.T]
    recomputed = 0
    for a in cases:
        lp, _ = qrcp.dgeqpf(a)
        order, free, mx, tk, rec = qrcp.dgeqpf_port(np.asfortranarray(a.copy()))
        assert np.array_equal(lp[:len(order)], order)
        assert np.array_equal(order, free) and np.array_equal(mx, tk)
        recomputed += rec
    assert recomputed > 0


def test_dgeqpf_recomputes_where_the_downdate_would_pick_wrongly():
    """On the cancellation matrix the second pivot by downdated norms differs
    from the true largest residual; LAPACK (and the restatement) take the
    true one, i.e. they recompute (the newer test of LAPACK Working Note 176,
    not the older 1 + 0.05 temp (nu/nu0)^2 == 1 that would not fire here)."""
    a = _cancellation_matrix(0)
    lp, _ = qrcp.dgeqpf(a)
    q = a[:, 0] / np.linalg.norm(a[:, 0])
    true_res = np.linalg.norm(a - np.outer(q, q @ a), axis=0)
    true_res[0] = -1
    nu = np.linalg.norm(a, axis=0)
    dd = nu * np.sqrt(np.maximum(1 - ((q @ a) / nu) ** 2, 0))
    dd[0] = -1
    assert lp[1] == np.argmax(true_res) != np.argmax(dd)


def test_dgeqpf_port_follows_forced_pivots():
    """With a forced pivot the run continues from that choice: the steps
    before it are unchanged, the forced step reports dgeqpf's own choice."""
    a = _cancellation_matrix(2)
    order, free, _, _, _ = qrcp.dgeqpf_port(a.copy(order="F"), 10)
    forced = list(order[:3]) + [order[5]] + [-1] * 6
    o2, f2, mx2, tk2, _ = qrcp.dgeqpf_port(a.copy(order="F"), 10, forced)
    assert list(o2[:4]) == forced[:4]
    assert np.array_equal(f2[:3], order[:3]) and f2[3] == order[3] and tk2[3] <= mx2[3]
    assert np.array_equal(o2[4:], f2[4:])  # free choices after the forced step
    with pytest.raises(ValueError):
        qrcp.dgeqpf_port(a.copy(order="F"), 10, list(order[:3]) + [order[1]])
