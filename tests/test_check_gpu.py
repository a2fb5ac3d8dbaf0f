"""GPU check (cuFFT) against the reference's checkcode: the goldens hold the fit
and Coulomb errors the reference printed for its own theta; the GPU check run
on that same theta must reproduce them. Also the check inside ISDF()."""
import numpy as np
import pytest

from conftest import load_golden
from oracle import check as ocheck

import libisdf_b200 as isdf
from libisdf_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["small_s1s2", "small_mu0"])
def test_check_reproduces_reference_numbers(torch_cuda, name):
    torch = torch_cuda
    g = load_golden(name)
    a = (int(g["nocc"]), int(g["nv1"]), int(g["nc1"]), int(g["nv2"]), int(g["nc2"]))
    rk = int(g["rk_eff"])
    dom = isdf.Domain(length=tuple(g["length"]), num_grid=tuple(int(x) for x in g["ng"]))
    d_psi = torch.from_numpy(np.ascontiguousarray(g["psi"].T)).cuda()
    d_th = torch.from_numpy(np.ascontiguousarray(g["theta"].T)).cuda()
    th_before = d_th.clone()
    fe, ce = isdf.check(dom, d_psi, a[0], g["psi"].shape[1], *a[1:], rk, g["piv"], d_th)
    assert torch.equal(d_th, th_before)  # theta is read only
    assert abs(fe / float(g["fit_err"]) - 1) < 1e-9
    # the Coulomb error is a small difference of large sums: 1e-6 relative
    assert abs(ce / float(g["coul_err"]) - 1) < 1e-6


def test_check_inside_isdf_si8(torch_cuda):
    """Si8-like shape (40^3 grid, 32 states, mu = 320), check = true: the
    report carries both errors, equal to the numpy restatement's on the same
    theta."""
    torch = torch_cuda
    s = synth.SI8
    psi = synth.shape_orbitals(s, 0)
    dom = isdf.Domain(length=(s.length,) * 3, num_grid=(s.n,) * 3)
    d_psi = torch.from_numpy(np.ascontiguousarray(psi.T)).cuda()
    d_theta = torch.empty((s.mu, s.ng), dtype=torch.float64, device="cuda")
    piv = np.zeros(s.ng, dtype=np.int32)
    rep = isdf.ISDF(d_psi, dom, s.nocc, s.nstate, s.nv1, s.nc1, s.nv2, s.nc2, s.mu, d_theta, piv,
                    s.kmeans_iters, check=True)
    th = np.asfortranarray(d_theta.cpu().numpy().T)
    fe, ce = ocheck.check(psi, (s.n,) * 3, (s.length,) * 3, s.nocc, s.nv1, s.nc1, s.nv2, s.nc2,
                          rep.rk_eff, piv, th)
    assert rep.fit_err > 0 and rep.coul_err > 0
    assert abs(rep.fit_err / fe - 1) < 1e-8
    assert abs(rep.coul_err / ce - 1) < 1e-6
