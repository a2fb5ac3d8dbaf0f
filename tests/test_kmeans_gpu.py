"""K-means selection on the GPU against the reference (bit-exact weight, piv,
effective mu and iteration count)."""
import numpy as np
import pytest

from conftest import load_golden, record_parity
from oracle import port

import libisdf_b200 as isdf
from libisdf_b200 import synth

pytestmark = pytest.mark.gpu
CASES = ["si8_example", "small_s1s2", "small_mu0", "small_iters0", "small_early"]


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(np.asfortranarray(a).T)).cuda()


@pytest.mark.parametrize("name", CASES)
def test_weight_bit_exact(torch_cuda, name):
    torch = torch_cuda
    g = load_golden(name)
    psi = g["psi"]
    d_psi = _dev(torch, psi)
    d_w = torch.empty(psi.shape[0], dtype=torch.float64, device="cuda")
    isdf.kmeans_weight(d_psi, psi.shape[0], psi.shape[1], int(g["nocc"]), int(g["nv1"]),
                       int(g["nc1"]), int(g["nv2"]), int(g["nc2"]), d_w)
    torch.cuda.synchronize()
    assert np.array_equal(d_w.cpu().numpy(), g["weight"])


@pytest.mark.parametrize("name", CASES)
def test_select_matches_reference(torch_cuda, name):
    torch = torch_cuda
    g = load_golden(name)
    dom = isdf.Domain(length=tuple(g["length"]), num_grid=tuple(int(x) for x in g["ng"]))
    d_w = torch.from_numpy(g["weight"]).cuda()
    piv, rk, it, npt = isdf.kmeans_select(dom, d_w, int(g["rk_requested"]), int(g["iters"]),
                                          rand_seed=int(g["rand_seed"]))
    assert (rk, it) == (int(g["rk_eff"]), int(g["n_iter"]))
    assert np.array_equal(piv, g["piv"])


def test_select_si8_synthetic_matches_oracle(torch_cuda):
    """Si8-like shape: 40^3 grid, 32 states, mu = 320, 100 iterations."""
    torch = torch_cuda
    s = synth.SI8
    psi = synth.shape_orbitals(s, 0)
    ng, ln = (s.n,) * 3, (s.length,) * 3
    piv_o, rk_o, it_o, w_o = port.kmeans_piv(psi, ng, ln, s.nocc, s.nv1, s.nc1, s.nv2, s.nc2,
                                             s.mu, s.kmeans_iters)
    g = load_golden("si8_synth_seed0")
    if synth.sha256(psi) == str(g["psi_sha256"]):  # same bits as when the golden was made
        assert np.array_equal(piv_o, g["piv"]) and rk_o == int(g["rk_eff"])
    dom = isdf.Domain(length=ln, num_grid=ng)
    d_psi = _dev(torch, psi)
    d_theta = torch.empty((s.mu, s.ng), dtype=torch.float64, device="cuda")
    piv = np.zeros(s.ng, dtype=np.int32)
    rep = isdf.ISDF(d_psi, dom, s.nocc, s.nstate, s.nv1, s.nc1, s.nv2, s.nc2, s.mu, d_theta, piv,
                    s.kmeans_iters)
    assert rep.rk_eff == rk_o and rep.kmeans_iters == it_o
    assert np.array_equal(piv, piv_o)
    # zero-filled columns past the effective mu
    assert float(d_theta[rep.rk_eff:].abs().max().cpu()) == 0.0 if rep.rk_eff < s.mu else True


def test_select_is_repeatable(torch_cuda):
    torch = torch_cuda
    g = load_golden("small_s1s2")
    dom = isdf.Domain(length=tuple(g["length"]), num_grid=tuple(int(x) for x in g["ng"]))
    d_w = torch.from_numpy(g["weight"]).cuda()
    a = isdf.kmeans_select(dom, d_w, 40, 50)
    b = isdf.kmeans_select(dom, d_w, 40, 50)
    assert np.array_equal(a[0], b[0]) and a[1:] == b[1:]


@pytest.mark.parametrize("seed", [0, 1])
def test_select_heavy_zero_tail(torch_cuda, seed):
    """Half of the grid falls below the weight filter, so half of the K-means
    points are copies of grid point 0 (the reference's zero-initialised index
    tail), here carrying the largest weight: their cluster's fold is dominated
    by that repeated addition."""
    torch = torch_cuda
    rng = np.random.default_rng(seed)
    ng = (20, 21, 19)
    n = int(np.prod(ng))
    w = rng.uniform(0.1, 1.0, size=n) ** 3
    w[rng.random(n) < 0.5] = 1e-13
    w[0] = 1.7
    length = (9.5, 10.0, 9.0)
    piv_o, rk_o, it_o = port.kmeans(w, ng, length, 50, 30)
    piv, rk, it, npt = isdf.kmeans_select(isdf.Domain(length=length, num_grid=ng),
                                          torch.from_numpy(w).cuda(), 50, 30)
    assert npt < n / 2 + n / 10
    assert (rk, it) == (rk_o, it_o)
    assert np.array_equal(piv, piv_o)


@pytest.mark.parametrize("mu,seed", [(500, 3), (1, 4), (2000, 5)])
def test_select_random_weights(torch_cuda, mu, seed):
    """Random weights on an anisotropic grid: many centroids per cell ring,
    equal-distance ties between lattice points, the pruned search against
    the brute-force restatement."""
    torch = torch_cuda
    rng = np.random.default_rng(seed)
    ng = (30, 25, 20)
    n = int(np.prod(ng))
    w = rng.uniform(0.0, 1.0, size=n) ** 4
    length = (12.0, 7.5, 9.0)
    piv_o, rk_o, it_o = port.kmeans(w, ng, length, mu, 40)
    piv, rk, it, npt = isdf.kmeans_select(isdf.Domain(length=length, num_grid=ng),
                                          torch.from_numpy(w).cuda(), mu, 40)
    assert (rk, it) == (rk_o, it_o)
    assert np.array_equal(piv, piv_o)


def _perturbed_prev(g, seed=1):
    """Pivots of a previous solve on a slightly different weight (as an SCF
    loop's last iteration would have left them)."""
    ng = tuple(int(x) for x in g["ng"])
    ln = tuple(float(x) for x in g["length"])
    rng = np.random.default_rng(seed)
    w2 = np.abs(g["weight"] * (1 + 0.05 * rng.standard_normal(g["weight"].shape)))
    prev, _, _ = port.kmeans(w2, ng, ln, int(g["rk_requested"]), int(g["iters"]))
    return prev


@pytest.mark.parametrize("name", ["si8_example", "small_s1s2", "small_mu0", "small_iters0"])
def test_warm_start_matches_reference(torch_cuda, name):
    """K-means warm start (utility.cpp:725-749) through ISDF() with
    kmeans_warm_start: the same piv, effective mu, iteration count and number
    of reused pivots as the port, and as the reference's own KMEAN called
    with the same previous piv where the reference build is present."""
    torch = torch_cuda
    g = load_golden(name)
    ng = tuple(int(x) for x in g["ng"])
    ln = tuple(float(x) for x in g["length"])
    a = (int(g["nocc"]), int(g["nv1"]), int(g["nc1"]), int(g["nv2"]), int(g["nc2"]))
    mu, iters = int(g["rk_requested"]), int(g["iters"])
    prev = _perturbed_prev(g)
    piv_o, rk_o, it_o, used_o = port.kmeans_warm(g["weight"], ng, ln, mu, iters, prev)
    from oracle import ref

    if ref.available():
        r = ref.kmeans_warm(g["weight"], ng, ln, mu, iters, prev)
        assert np.array_equal(r[0], piv_o) and r[1:] == (rk_o, it_o, used_o)
    psi = g["psi"]
    d_psi = _dev(torch, psi)
    d_theta = torch.empty((mu, psi.shape[0]), dtype=torch.float64, device="cuda")
    piv = prev.copy()
    rep = isdf.ISDF(d_psi, isdf.Domain(length=ln, num_grid=ng), a[0], psi.shape[1], *a[1:], mu,
                    d_theta, piv, iters, options=isdf.Options(kmeans_warm_start=True))
    assert (rep.rk_eff, rep.kmeans_iters, rep.kmeans_warm_pivots) == (rk_o, it_o, used_o)
    assert np.array_equal(piv, piv_o)
    # without the option the caller's piv is ignored, as in the reference
    piv = prev.copy()
    rep = isdf.ISDF(d_psi, isdf.Domain(length=ln, num_grid=ng), a[0], psi.shape[1], *a[1:], mu,
                    d_theta, piv, iters)
    assert rep.kmeans_warm_pivots == -1 and np.array_equal(piv, g["piv"])


def test_warm_start_si8_perturbed_orbitals(torch_cuda):
    """An SCF-like step on the Si8-like shape: the orbitals change slightly
    between two solves; the second solve starts from the first one's piv and
    equals the port's warm start bit for bit."""
    torch = torch_cuda
    s = synth.SI8
    psi = synth.shape_orbitals(s, 0)
    rng = np.random.default_rng(9)
    psi2 = np.asfortranarray(np.linalg.qr(psi + 1e-3 * rng.standard_normal(psi.shape))[0])
    ng, ln = (s.n,) * 3, (s.length,) * 3
    a = (s.nocc, s.nv1, s.nc1, s.nv2, s.nc2)
    dom = isdf.Domain(length=ln, num_grid=ng)
    d_theta = torch.empty((s.mu, s.ng), dtype=torch.float64, device="cuda")
    piv = np.zeros(s.ng, dtype=np.int32)
    rep1 = isdf.ISDF(_dev(torch, psi), dom, s.nocc, s.nstate, *a[1:], s.mu, d_theta, piv,
                     s.kmeans_iters)
    prev = piv.copy()
    w2 = port.weight(psi2, *a)
    piv_o, rk_o, it_o, used_o = port.kmeans_warm(w2, ng, ln, s.mu, s.kmeans_iters, prev)
    cold = port.kmeans(w2, ng, ln, s.mu, s.kmeans_iters)
    rep2 = isdf.ISDF(_dev(torch, psi2), dom, s.nocc, s.nstate, *a[1:], s.mu, d_theta, piv,
                     s.kmeans_iters, options=isdf.Options(kmeans_warm_start=True))
    assert (rep2.rk_eff, rep2.kmeans_iters, rep2.kmeans_warm_pivots) == (rk_o, it_o, used_o)
    assert np.array_equal(piv, piv_o)
    record_parity("K-means warm start Si8-like", "Lloyd iterations warm / cold",
                  f"{rep2.kmeans_iters} / {cold[2]} (first solve {rep1.kmeans_iters})")


def test_batched_selection_matches_reference(torch_cuda):
    """The batched selection of small systems (one cooperative launch, a CTA
    group per system, the serving loop's path for small requests): every
    result equals the reference's (goldens: piv, effective mu, iteration
    count, including the npt < mu early return) and, for the Si8-like system
    and a random-weight grid, the port's, in one batch of mixed sizes."""
    torch = torch_cuda
    names = ["si8_example", "small_s1s2", "small_mu0", "small_iters0", "small_early"]
    doms, ws, mus, its, want = [], [], [], [], []
    for name in names:
        g = load_golden(name)
        doms.append(isdf.Domain(length=tuple(g["length"]), num_grid=tuple(int(x) for x in g["ng"])))
        ws.append(torch.from_numpy(g["weight"]).cuda())
        mus.append(int(g["rk_requested"]))
        its.append(int(g["iters"]))
        want.append((g["piv"], int(g["rk_eff"]), int(g["n_iter"])))
    s = synth.SI8
    psi = synth.shape_orbitals(s, 0)
    w8 = port.weight(psi, s.nocc, s.nv1, s.nc1, s.nv2, s.nc2)
    p8, r8, i8 = port.kmeans(w8, (s.n,) * 3, (s.length,) * 3, s.mu, s.kmeans_iters)
    doms.append(isdf.Domain(length=(s.length,) * 3, num_grid=(s.n,) * 3))
    ws.append(torch.from_numpy(w8).cuda())
    mus.append(s.mu)
    its.append(s.kmeans_iters)
    want.append((p8, r8, i8))
    rng = np.random.default_rng(3)
    ng = (30, 25, 20)
    wr = rng.uniform(0.0, 1.0, size=int(np.prod(ng))) ** 4
    pr, rr, ir = port.kmeans(wr, ng, (12.0, 7.5, 9.0), 500, 40)
    doms.append(isdf.Domain(length=(12.0, 7.5, 9.0), num_grid=ng))
    ws.append(torch.from_numpy(wr).cuda())
    mus.append(500)
    its.append(40)
    want.append((pr, rr, ir))
    got = isdf.kmeans_select_batch(doms, ws, mus, its, rand_seed=1)
    for k, ((piv, rk, it, _), (wp, wr_, wi)) in enumerate(zip(got, want)):
        assert (rk, it) == (wr_, wi), k
        assert np.array_equal(piv, wp), k
