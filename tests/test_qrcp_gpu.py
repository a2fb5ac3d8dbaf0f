"""QRCP selection on the GPU against the restatement of getpoints_QRCP with
LAPACK dgeqpf (the reference calls ScaLAPACK pdgeqpf, which cannot be built
here). The first mu pivots are compared; a mismatch is accepted only where the
two candidate columns' residual norms tie to 1e-9 relative (a near-tie that
rounding legitimately decides either way) or where both residuals are at
roundoff level, below 1e-10 of the largest column norm (the sketched pair
space is exhausted: the reference's own Si8 example has 16 states, so at most
136 independent pair products), and nothing after it is compared."""
import numpy as np
import pytest

from conftest import load_golden
from oracle import fit as ofit
from oracle import qrcp

import libisdf_b200 as isdf
from libisdf_b200 import synth

pytestmark = pytest.mark.gpu


def _gpu_qrcp(torch, psi, ng, length, a, mu, factor, seed):
    d_psi = torch.from_numpy(np.ascontiguousarray(psi.T)).cuda()
    d_theta = torch.zeros((mu, psi.shape[0]), dtype=torch.float64, device="cuda")
    piv = np.zeros(psi.shape[0], dtype=np.int32)
    opts = isdf.Options(qrcp_oversample=factor, qrcp_seed=seed)
    rep = isdf.ISDF(d_psi, isdf.Domain(length=length, num_grid=ng), a[0], psi.shape[1], a[1],
                    a[2], a[3], a[4], mu, d_theta, piv, 10, s1="QRCP", options=opts)
    return piv, np.asfortranarray(d_theta.cpu().numpy().T), rep


def _check_pivots(psi, a, mu, factor, seed, piv_gpu):
    piv_o, ntot, piv_mg, idx, _ = qrcp.select(psi, *a, mu, seed=seed, factor=factor)
    k = min(mu, ntot, qrcp.num_pre(mu, factor) ** 2)
    same = piv_gpu[:k] == piv_o[:k]
    if same.all():
        return k, k
    first = int(np.argmin(same))
    # near-tie check at the first difference
    p = qrcp.num_pre(mu, factor)
    g1, g2 = qrcp.sketch(a[1] + a[2], a[3] + a[4], p, seed)
    A = psi[:, a[0] - a[1]:a[0] + a[2]] @ g1
    B = psi[:, a[0] - a[3]:a[0] + a[4]] @ g2
    cols = np.array([piv_o[first], piv_gpu[first]])
    sel = piv_o[:first]
    def feat(r):
        return (B[r][:, None, :] * A[r][:, :, None]).reshape(len(r), p * p).T
    res = qrcp.residual_norms(feat(np.concatenate([sel, cols])), np.arange(len(sel)))
    r_o, r_g = res[-2], res[-1]
    top = np.sqrt(qrcp.mg_norms(A, B).max())
    assert (abs(r_o - r_g) <= 1e-9 * max(r_o, r_g) or max(r_o, r_g) <= 1e-10 * top), \
        (first, r_o, r_g, top)
    return k, k


@pytest.mark.parametrize("name,mu,factor,seed", [("small_s1s2", 16, 1.5, 41),
                                                 ("small_mu0", 16, 2.5, 2),
                                                 ("si8_example", 160, 1.5, 41)])
def test_qrcp_pivots_match_oracle(torch_cuda, name, mu, factor, seed):
    g = load_golden(name)
    a = (int(g["nocc"]), int(g["nv1"]), int(g["nc1"]), int(g["nv2"]), int(g["nc2"]))
    ng = tuple(int(x) for x in g["ng"])
    piv, th, rep = _gpu_qrcp(torch_cuda, g["psi"], ng, tuple(g["length"]), a, mu, factor, seed)
    agree, k = _check_pivots(g["psi"], a, mu, factor, seed, piv)
    assert agree == k
    # theta from these pivots against the numpy fit
    th_o = ofit.getbasis(g["psi"], *a, mu, piv)
    fd = ofit.fitted_densities(th, g["psi"], *a, mu, piv)
    fd_o = ofit.fitted_densities(th_o, g["psi"], *a, mu, piv)
    assert ofit.rel(fd, fd_o) <= 1e-9


def test_qrcp_si8_synthetic(torch_cuda):
    """Si8-like shape with the QRCP selector (40^3, 32 states, mu = 320)."""
    s = synth.SI8
    psi = synth.shape_orbitals(s, 2)
    a = (s.nocc, s.nv1, s.nc1, s.nv2, s.nc2)
    piv, th, rep = _gpu_qrcp(torch_cuda, psi, (s.n,) * 3, (s.length,) * 3, a, s.mu, 2.5, 2)
    agree, k = _check_pivots(psi, a, s.mu, 2.5, 2, piv)
    assert agree >= min(k, 64)
