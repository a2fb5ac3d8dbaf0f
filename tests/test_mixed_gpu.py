"""Mixed-precision form (INT8-sliced tcgen05 GEMMs, FP64 Cholesky and
triangular inverse) against the FP64 form and the FP64 oracle. The bar is
the mixed form's accuracy target: fitted pair densities (theta C) within 1e-6 relative of the
FP64 result; piv is identical (K-means stays FP64)."""
import numpy as np
import pytest

from conftest import load_golden
from oracle import fit as ofit

import libisdf_b200 as isdf
from libisdf_b200 import synth

pytestmark = pytest.mark.gpu


def _solve(torch, psi, shape_args, mu, iters, dom, precision, slices=6):
    nocc, nv1, nc1, nv2, nc2 = shape_args
    d_psi = torch.from_numpy(np.ascontiguousarray(psi.T)).cuda()
    d_theta = torch.empty((mu, psi.shape[0]), dtype=torch.float64, device="cuda")
    piv = np.zeros(psi.shape[0], dtype=np.int32)
    rep = isdf.ISDF(d_psi, dom, nocc, psi.shape[1], nv1, nc1, nv2, nc2, mu, d_theta, piv, iters,
                    options=isdf.Options(precision=precision, mixed_slices=slices))
    return piv, np.asfortranarray(d_theta.cpu().numpy().T), rep


@pytest.mark.parametrize("slices", [6, 7])
def test_mixed_si8_against_fp64(torch_cuda, slices):
    s = synth.SI8
    psi = synth.shape_orbitals(s, 0)
    a = (s.nocc, s.nv1, s.nc1, s.nv2, s.nc2)
    dom = isdf.Domain(length=(s.length,) * 3, num_grid=(s.n,) * 3)
    piv64, th64, r64 = _solve(torch_cuda, psi, a, s.mu, s.kmeans_iters, dom, isdf.PRECISION_FP64)
    pivm, thm, rm = _solve(torch_cuda, psi, a, s.mu, s.kmeans_iters, dom, isdf.PRECISION_MIXED,
                           slices)
    assert np.array_equal(piv64, pivm) and r64.rk_eff == rm.rk_eff
    rk = rm.rk_eff
    rows = np.arange(0, s.ng, 3)
    fd64 = \
        ofit.fitted_densities(th64, psi, *a, rk, piv64, rows)
    fdm = ofit.fitted_densities(thm, psi, *a, rk, pivm, rows)
    err = ofit.rel(fdm, fd64)
    assert err <= 1e-6, err
    # and against the FP64 oracle's theta
    th_o = ofit.getbasis(psi, *a, rk, piv64)
    assert ofit.rel(fdm, ofit.fitted_densities(th_o, psi, *a, rk, piv64, rows)) <= 1e-6


def test_mixed_s1_ne_s2(torch_cuda):
    g = load_golden("small_s1s2")
    a = (int(g["nocc"]), int(g["nv1"]), int(g["nc1"]), int(g["nv2"]), int(g["nc2"]))
    rk = int(g["rk_eff"])
    d_psi = torch_cuda.from_numpy(np.ascontiguousarray(g["psi"].T)).cuda()
    d_th = torch_cuda.zeros((rk, g["psi"].shape[0]), dtype=torch_cuda.float64, device="cuda")
    assert isdf.fit(d_psi, g["psi"].shape[0], g["psi"].shape[1], *a, rk, g["piv"], d_th,
                    precision=isdf.PRECISION_MIXED) == 0
    th = np.asfortranarray(d_th.cpu().numpy().T)
    fd = ofit.fitted_densities(th, g["psi"], *a, rk, g["piv"])
    fd_ref = ofit.fitted_densities(g["theta"], g["psi"], *a, rk, g["piv"])
    assert ofit.rel(fd, fd_ref) <= 1e-6
