"""QRCP selection on the GPU against the restatement of getpoints_QRCP with the
column-pivoted QR of LAPACK dgeqpf (the reference calls ScaLAPACK pdgeqpf,
which cannot be built here; oracle/qrcp_port.cpp restates dgeqpf and is pinned
to OpenBLAS's dgeqpf in tests/test_qrcp.py).

Every pivot is checked. The oracle runs dgeqpf on the reference's MG matrix
but takes, at each step, the grid point the GPU took, and reports the point
dgeqpf itself would have taken there. A step passes when the two agree, or
when the GPU's point ties dgeqpf's to NEAR_TIE relative in dgeqpf's own
(downdated or recomputed) norms - rounding legitimately decides such a tie
either way, and the comparison continues from the GPU's choice - or when the
remaining residuals are at roundoff level, below 1e-10 of the largest column
norm (the sketched pair space is exhausted: the reference's own Si8 example
has 16 states, so at most 136 independent pair products)."""
import numpy as np
import pytest

from conftest import load_golden, record_parity
from oracle import fit as ofit
from oracle import qrcp

import libisdf_b200 as isdf
from libisdf_b200 import synth

pytestmark = pytest.mark.gpu

NEAR_TIE = 1e-8


def _gpu_qrcp(torch, psi, ng, length, a, mu, factor, seed):
    d_psi = torch.from_numpy(np.ascontiguousarray(psi.T)).cuda()
    d_theta = torch.zeros((mu, psi.shape[0]), dtype=torch.float64, device="cuda")
    piv = np.zeros(psi.shape[0], dtype=np.int32)
    opts = isdf.Options(qrcp_oversample=factor, qrcp_seed=seed)
    rep = isdf.ISDF(d_psi, isdf.Domain(length=length, num_grid=ng), a[0], psi.shape[1], a[1],
                    a[2], a[3], a[4], mu, d_theta, piv, 10, s1="QRCP", options=opts)
    return piv, np.asfortranarray(d_theta.cpu().numpy().T), rep


def check_all_pivots(tag, psi, a, mu, factor, seed, piv_gpu, steps_gpu, kmax=None):
    """Checks every GPU pivot against dgeqpf following the GPU's sequence;
    returns the number of steps checked."""
    free, mx, tk, k, top, rec = qrcp.follow_pivots(psi, *a, mu, piv_gpu, seed=seed,
                                                   factor=factor, kmax=kmax)
    assert steps_gpu >= k
    same = free == piv_gpu[:k]
    gap = (mx - tk) / np.maximum(mx, np.finfo(float).tiny)
    exhausted = mx <= 1e-10 * top
    ok = same | (gap <= NEAR_TIE) | exhausted
    bad = np.nonzero(~ok)[0]
    assert bad.size == 0, (f"step {bad[0]}: GPU took {piv_gpu[bad[0]]}, dgeqpf {free[bad[0]]}, "
                           f"norms {tk[bad[0]]:.17g} vs {mx[bad[0]]:.17g}")
    ties = ~same & ~exhausted
    record_parity(tag, "pivots equal to dgeqpf's own choice", f"{int(same.sum())}/{k}")
    record_parity(tag, "largest near-tie gap taken", float(gap[ties].max()) if ties.any() else 0.0,
                  NEAR_TIE)
    record_parity(tag, "oracle norm recomputes", rec)
    return k


@pytest.mark.parametrize("name,mu,factor,seed", [("small_s1s2", 16, 1.5, 41),
                                                 ("small_mu0", 16, 2.5, 2),
                                                 ("si8_example", 160, 1.5, 41)])
def test_qrcp_pivots_match_oracle(torch_cuda, name, mu, factor, seed):
    g = load_golden(name)
    a = (int(g["nocc"]), int(g["nv1"]), int(g["nc1"]), int(g["nv2"]), int(g["nc2"]))
    ng = tuple(int(x) for x in g["ng"])
    piv, th, rep = _gpu_qrcp(torch_cuda, g["psi"], ng, tuple(g["length"]), a, mu, factor, seed)
    k = check_all_pivots(f"qrcp {name}", g["psi"], a, mu, factor, seed, piv, rep.qrcp_steps)
    assert k == min(mu, rep.npt, qrcp.num_pre(mu, factor) ** 2)
    if name == "si8_example":  # rank exhausted: the downdate loses accuracy, norms recomputed
        assert rep.qrcp_norm_recomputes > 0
    record_parity(f"qrcp {name}", "GPU norm recomputes", rep.qrcp_norm_recomputes)
    # theta from these pivots against the numpy fit
    th_o = ofit.getbasis(g["psi"], *a, mu, piv)
    fd = ofit.fitted_densities(th, g["psi"], *a, mu, piv)
    fd_o = ofit.fitted_densities(th_o, g["psi"], *a, mu, piv)
    err = ofit.rel(fd, fd_o)
    record_parity(f"qrcp {name}", "fitted densities vs oracle", err, 1e-10)
    assert err <= 1e-10


def test_qrcp_si8_synthetic(torch_cuda):
    """Si8-like shape with the QRCP selector (40^3, 32 states, mu = 320,
    oversampling 2.5, seed 2): all 320 pivots."""
    s = synth.SI8
    psi = synth.shape_orbitals(s, 2)
    a = (s.nocc, s.nv1, s.nc1, s.nv2, s.nc2)
    piv, th, rep = _gpu_qrcp(torch_cuda, psi, (s.n,) * 3, (s.length,) * 3, a, s.mu, 2.5, 2)
    k = check_all_pivots("qrcp Si8-like", psi, a, s.mu, 2.5, 2, piv, rep.qrcp_steps)
    assert k == s.mu
    rows = np.arange(0, s.ng, 7)
    fd = ofit.fitted_densities(th, psi, *a, s.mu, piv, rows)
    fd_o = ofit.fitted_densities(ofit.getbasis_rows(psi, *a, s.mu, piv, rows), psi, *a, s.mu,
                                 piv)
    err = ofit.rel(fd, fd_o)
    record_parity("qrcp Si8-like", "fitted densities vs oracle", err, 1e-10)
    assert err <= 1e-10
