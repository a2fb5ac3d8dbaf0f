"""Parity at the benchmark sizes (the shapes bench.py quotes):

  * Si64-like K-means (80^3 grid, 256 states, mu = 2048, 100 iterations,
    seed 1): piv, the effective mu and the iteration count bit-exact against
    the K-means port (oracle/kmeans_port.cpp, pinned to the reference's own
    KMEAN), with the pruned cell search fully exercised; theta of the FP64 and
    of the mixed form against the oracle fit on sampled grid rows;
  * Si64-like QRCP (oversampling 2.5, seed 2): a prefix of the pivots checked
    step by step against dgeqpf on the reference's MG matrix, theta against
    the oracle on sampled rows;
  * Si64-like valence x conduction (S1 = 128 occupied, S2 = 128 empty states,
    mu = 1024): the same checks on the two-factor (S1 != S2) path;
  * Si216-like (108^3, 864 states, mu = 4320, seed 3): the mixed form's and the
    FP64 form's theta against the oracle fit on sampled rows.

theta is compared on 2048 sampled grid rows (oracle.fit.getbasis_rows computes
exactly those rows of the full-size fit) and the fitted pair densities theta C
on 1024 sampled state pairs. Bounds: the mixed form's fitted densities within
1e-6 of the oracle (the mixed form's accuracy target); the FP64 form's within
max(1e-10, 20 x the distance between two correct FP64 CPU solutions of the
same rows, Cholesky + triangular solves vs LU): at cond(C C^T) ~ 1e10 FP64
rounding alone moves the fitted densities far more than 1e-10, and the test
records that spread beside the GPU's difference."""
import numpy as np
import pytest

from conftest import record_parity
from oracle import fit as ofit
from oracle import port
from oracle import qrcp

import libisdf_b200 as isdf
from libisdf_b200 import synth

pytestmark = pytest.mark.gpu

ROWS, PAIRS = 2048, 1024


def _sample(shape, seed=0):
    rng = np.random.default_rng(seed)
    rows = np.sort(rng.choice(shape.ng, size=ROWS, replace=False))
    i = shape.nocc - shape.nv1 + rng.integers(0, shape.nv1 + shape.nc1, size=PAIRS)
    j = shape.nocc - shape.nv2 + rng.integers(0, shape.nv2 + shape.nc2, size=PAIRS)
    return rows, i, j


def _theta_rows(torch, d_theta, rk, rows):
    idx = torch.from_numpy(rows).cuda()
    return d_theta[:rk].index_select(1, idx).T.cpu().numpy()


def _fd(th_rows, psi, piv, rk, i, j):
    pm = psi[np.asarray(piv[:rk], dtype=np.int64)]
    return th_rows[:, :rk] @ (pm[:, i] * pm[:, j])


def _solve(torch, d_psi, shape, d_theta, piv, options, s1="Kmeans"):
    dom = isdf.Domain(length=(shape.length,) * 3, num_grid=(shape.n,) * 3)
    rep = isdf.ISDF(d_psi, dom, shape.nocc, shape.nstate, shape.nv1, shape.nc1, shape.nv2,
                    shape.nc2, shape.mu, d_theta, piv, shape.kmeans_iters, s1=s1,
                    options=options)
    torch.cuda.synchronize()
    return rep


def _spread(tag, psi, a, piv, rk, rows, th_o, pi, pj):
    """Fitted-density bound for the FP64 form: max(1e-10, 20 x the distance
    between the oracle's Cholesky solve and an LU solve of the same rows)."""
    th_lu = ofit.getbasis_rows(psi, *a, rk, piv, rows, solver="lu")
    spread = ofit.rel(_fd(th_lu, psi, piv, rk, pi, pj), _fd(th_o, psi, piv, rk, pi, pj))
    record_parity(tag, "fitted densities: CPU Cholesky vs CPU LU (sampled)", spread)
    record_parity(tag, "theta: CPU Cholesky vs CPU LU (sampled rows)", ofit.rel(th_lu, th_o))
    return max(1e-10, 20 * spread)


def _compare(tag, th_rows, th_o, psi, piv, rk, pi, pj, fd_bound):
    fd, fd_o = _fd(th_rows, psi, piv, rk, pi, pj), _fd(th_o, psi, piv, rk, pi, pj)
    e_fd, e_th = ofit.rel(fd, fd_o), ofit.rel(th_rows[:, :rk], th_o)
    record_parity(tag, "fitted densities vs oracle (sampled)", e_fd, fd_bound)
    record_parity(tag, "theta vs oracle (sampled rows)", e_th)
    assert e_fd <= fd_bound, (tag, e_fd)
    return e_fd


def test_si64_kmeans_piv_bit_exact_and_theta(torch_cuda):
    torch = torch_cuda
    s = synth.SI64
    psi = synth.shape_orbitals(s, 1, device="cuda")
    a = (s.nocc, s.nv1, s.nc1, s.nv2, s.nc2)
    piv_o, rk_o, it_o, _ = port.kmeans_piv(psi, (s.n,) * 3, (s.length,) * 3, *a, s.mu,
                                           s.kmeans_iters)
    d_psi = torch.from_numpy(np.ascontiguousarray(psi.T)).cuda()
    d_theta = torch.empty((s.mu, s.ng), dtype=torch.float64, device="cuda")
    piv = np.zeros(s.ng, dtype=np.int32)
    rep = _solve(torch, d_psi, s, d_theta, piv, isdf.Options())
    record_parity("Si64 K-means", "rk_eff / iterations (GPU, port)",
                  f"{rep.rk_eff}/{rep.kmeans_iters}, {rk_o}/{it_o}")
    assert (rep.rk_eff, rep.kmeans_iters) == (rk_o, it_o)
    assert np.array_equal(piv, piv_o), int(np.argmax(piv != piv_o))
    assert rep.kmeans_search_frac < 1.0  # the pruned search skipped work
    rows, pi, pj = _sample(s)
    th_o = ofit.getbasis_rows(psi, *a, rk_o, piv_o, rows)
    bound = _spread("Si64 K-means", psi, a, piv_o, rk_o, rows, th_o, pi, pj)
    _compare("Si64 FP64", _theta_rows(torch, d_theta, rk_o, rows), th_o, psi, piv_o, rk_o, pi,
             pj, bound)
    rep_m = _solve(torch, d_psi, s, d_theta, piv, isdf.Options(precision=isdf.PRECISION_MIXED))
    assert rep_m.rk_eff == rk_o and np.array_equal(piv, piv_o)
    _compare("Si64 mixed", _theta_rows(torch, d_theta, rk_o, rows), th_o, psi, piv_o, rk_o, pi,
             pj, 1e-6)


def test_si64_valence_conduction(torch_cuda):
    """S1 != S2 at the Si64 size (the two-factor epilogues): the valence x
    conduction window of 128 occupied x 128 empty states (mu = 1024), the pair
    products a GW / BSE code fits. piv, the effective mu and the iteration
    count bit-exact against the K-means port with the same window; theta of the
    FP64 and of the mixed form against the oracle on sampled rows and pairs."""
    torch = torch_cuda
    s = synth.SI64VC
    psi = synth.shape_orbitals(s, 1, device="cuda")
    a = (s.nocc, s.nv1, s.nc1, s.nv2, s.nc2)
    piv_o, rk_o, it_o, _ = port.kmeans_piv(psi, (s.n,) * 3, (s.length,) * 3, *a, s.mu,
                                           s.kmeans_iters)
    d_psi = torch.from_numpy(np.ascontiguousarray(psi.T)).cuda()
    d_theta = torch.empty((s.mu, s.ng), dtype=torch.float64, device="cuda")
    piv = np.zeros(s.ng, dtype=np.int32)
    rep = _solve(torch, d_psi, s, d_theta, piv, isdf.Options())
    record_parity("Si64 valence x conduction", "rk_eff / iterations (GPU, port)",
                  f"{rep.rk_eff}/{rep.kmeans_iters}, {rk_o}/{it_o}")
    assert (rep.rk_eff, rep.kmeans_iters) == (rk_o, it_o)
    assert np.array_equal(piv, piv_o), int(np.argmax(piv != piv_o))
    rows, pi, pj = _sample(s)
    th_o = ofit.getbasis_rows(psi, *a, rk_o, piv_o, rows)
    bound = _spread("Si64 valence x conduction", psi, a, piv_o, rk_o, rows, th_o, pi, pj)
    _compare("Si64 valence x conduction FP64", _theta_rows(torch, d_theta, rk_o, rows), th_o, psi,
             piv_o, rk_o, pi, pj, bound)
    rep_m = _solve(torch, d_psi, s, d_theta, piv, isdf.Options(precision=isdf.PRECISION_MIXED))
    assert rep_m.rk_eff == rk_o and np.array_equal(piv, piv_o)
    _compare("Si64 valence x conduction mixed", _theta_rows(torch, d_theta, rk_o, rows), th_o,
             psi, piv_o, rk_o, pi, pj, 1e-6)


def test_si64_qrcp_pivots_and_theta(torch_cuda):
    """Config 2: the QRCP selector with oversampling 2.5 and seed 2. dgeqpf on
    the 5184 x 305087 MG matrix costs ~0.3 s of host time per step, so the
    first 96 pivots are checked step by step (each against dgeqpf following
    the GPU's earlier choices)."""
    torch = torch_cuda
    from test_qrcp_gpu import check_all_pivots

    s = synth.SI64
    psi = synth.shape_orbitals(s, 1, device="cuda")
    a = (s.nocc, s.nv1, s.nc1, s.nv2, s.nc2)
    d_psi = torch.from_numpy(np.ascontiguousarray(psi.T)).cuda()
    d_theta = torch.empty((s.mu, s.ng), dtype=torch.float64, device="cuda")
    piv = np.zeros(s.ng, dtype=np.int32)
    rep = _solve(torch, d_psi, s, d_theta, piv,
                 isdf.Options(qrcp_oversample=2.5, qrcp_seed=2), s1="QRCP")
    assert rep.qrcp_steps == s.mu and qrcp.num_pre(s.mu, 2.5) == 72
    record_parity("Si64 QRCP", "GPU norm recomputes", rep.qrcp_norm_recomputes)
    rows, pi, pj = _sample(s)
    th_o = ofit.getbasis_rows(psi, *a, s.mu, piv, rows)
    bound = _spread("Si64 QRCP", psi, a, piv, s.mu, rows, th_o, pi, pj)
    _compare("Si64 QRCP FP64", _theta_rows(torch, d_theta, s.mu, rows), th_o, psi, piv, s.mu, pi,
             pj, bound)
    del d_theta
    torch.cuda.empty_cache()
    k = check_all_pivots("Si64 QRCP", psi, a, s.mu, 2.5, 2, piv, rep.qrcp_steps, kmax=96)
    assert k == 96


def test_si216_mixed_and_fp64_vs_oracle(torch_cuda):
    torch = torch_cuda
    s = synth.SI216
    psi = synth.shape_orbitals(s, 3, device="cuda")
    a = (s.nocc, s.nv1, s.nc1, s.nv2, s.nc2)
    d_psi = torch.from_numpy(np.ascontiguousarray(psi.T)).cuda()
    d_theta = torch.empty((s.mu, s.ng), dtype=torch.float64, device="cuda")
    piv = np.zeros(s.ng, dtype=np.int32)
    rep = _solve(torch, d_psi, s, d_theta, piv, isdf.Options(precision=isdf.PRECISION_MIXED))
    rk = rep.rk_eff
    rows, pi, pj = _sample(s)
    th_m = _theta_rows(torch, d_theta, rk, rows)
    piv_m = piv[:rk].copy()
    rep_f = _solve(torch, d_psi, s, d_theta, piv, isdf.Options())
    assert rep_f.rk_eff == rk and np.array_equal(piv[:rk], piv_m)
    th_f = _theta_rows(torch, d_theta, rk, rows)
    del d_theta
    torch.cuda.empty_cache()
    th_o = ofit.getbasis_rows(psi, *a, rk, piv_m, rows)
    _compare("Si216 mixed", th_m, th_o, psi, piv_m, rk, pi, pj, 1e-6)
    bound = _spread("Si216", psi, a, piv_m, rk, rows, th_o, pi, pj)
    _compare("Si216 FP64", th_f, th_o, psi, piv_m, rk, pi, pj, bound)
