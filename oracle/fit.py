"""Test infrastructure only (oracle): numpy restatement of the FP64 ISDF fit.

Follows src/cpu/getbasis_MPI.cpp:9-250 (the CPU twin of the GPU fit in
src/cuda/isdf-gpu.cpp:112-402) at one rank:
  * psi(mu) gather                       getbasis_MPI.cpp:61-116
  * P = psi_S1 psi_S1(mu)^T (and P2)      :122-141, :163-167
  * Z C^T = P1 o P2  (P1 o P1 if S1 = S2) :146-152, :173-179
  * C C^T(mu, nu) = Z C^T(piv_nu, mu)     :188-214
  * eps = 1e-10 * (trace / rk)            :222-231
  * lower Cholesky                        :234
  * theta L^T = Z C^T, theta L = (that)   :239-240
Only tests, the smoke check and bench.py's CPU-baseline leg import this.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sl


def zct(psi, nocc, nv1, nc1, nv2, nc2, rk, piv):
    psi = np.asarray(psi)
    p = np.asarray(piv[:rk], dtype=np.int64)
    s1 = slice(nocc - nv1, nocc + nc1)
    s2 = slice(nocc - nv2, nocc + nc2)
    p1 = psi[:, s1] @ psi[p, s1].T
    if nv1 != nv2 or nc1 != nc2:
        return p1 * (psi[:, s2] @ psi[p, s2].T)
    return p1 * p1


def cct(z, rk, piv):
    p = np.asarray(piv[:rk], dtype=np.int64)
    cc = np.array(z[p, :].T, order="F")  # cc[mu, nu] = z[piv[nu], mu]
    tr = 0.0
    for i in range(rk):  # sequential trace, as the reference loops
        tr += cc[i, i]
    eps = 1e-10 * (tr / float(rk))
    cc[np.diag_indices(rk)] += eps
    return cc, eps


def getbasis(psi, nocc, nv1, nc1, nv2, nc2, rk, piv):
    """theta (Ng x rk, F-order)."""
    z = zct(psi, nocc, nv1, nc1, nv2, nc2, rk, piv)
    cc, _ = cct(z, rk, piv)
    L = np.linalg.cholesky(cc)
    y = sl.solve_triangular(L, z.T, lower=True)          # L y = z^T  <=>  y^T L^T = z
    th = sl.solve_triangular(L, y, lower=True, trans="T")  # L^T t = y  <=>  t^T L = y^T
    return np.asfortranarray(th.T)


def getbasis_rows(psi, nocc, nv1, nc1, nv2, nc2, rk, piv, rows, solver="cholesky"):
    """theta restricted to the grid rows `rows` (len(rows) x rk): the same
    operations as getbasis, but Z C^T is formed only on those rows and on the
    rk interpolation rows that C C^T is gathered from (getbasis_MPI.cpp:188-214).
    Each row of theta depends only on its own row of Z C^T, so this is the
    full-size fit evaluated where it is compared, at a cost independent of Ng.
    solver="lu" solves the same system by LU instead of Cholesky and two
    triangular solves: a second correct FP64 ordering, whose distance from the
    first measures how far FP64 rounding alone moves the result."""
    psi = np.asarray(psi)
    p = np.asarray(piv[:rk], dtype=np.int64)
    rows = np.asarray(rows, dtype=np.int64)
    s1 = slice(nocc - nv1, nocc + nc1)
    s2 = slice(nocc - nv2, nocc + nc2)

    def z(r):
        p1 = psi[r][:, s1] @ psi[p][:, s1].T
        if nv1 != nv2 or nc1 != nc2:
            return p1 * (psi[r][:, s2] @ psi[p][:, s2].T)
        return p1 * p1

    # Z C^T on the interpolation rows: row j is grid row piv[j], so C C^T
    # gathers cc[mu, nu] = zp[nu, mu]
    cc, _ = cct(z(p), rk, np.arange(rk))
    zr = z(rows)
    if solver == "lu":
        return np.asfortranarray(sl.solve(cc.T, zr.T, assume_a="gen").T)
    L = np.linalg.cholesky(cc)
    y = sl.solve_triangular(L, zr.T, lower=True)
    th = sl.solve_triangular(L, y, lower=True, trans="T")
    return np.asfortranarray(th.T)


def pair_densities(psi_rows, nocc, nv1, nc1, nv2, nc2):
    """rho_ij on the given rows, column (k - lo1) * n2 + (j - lo2), as checkcode.cpp:62-73."""
    a = psi_rows[:, nocc - nv1:nocc + nc1]
    b = psi_rows[:, nocc - nv2:nocc + nc2]
    return (a[:, :, None] * b[:, None, :]).reshape(psi_rows.shape[0], -1)


def fitted_densities(theta, psi, nocc, nv1, nc1, nv2, nc2, rk, piv, rows=None):
    """theta C restricted to `rows` (all when None): the fitted pair densities."""
    c = pair_densities(np.asarray(psi)[np.asarray(piv[:rk], dtype=np.int64)], nocc, nv1, nc1,
                       nv2, nc2)
    th = theta if rows is None else theta[rows]
    return th[:, :rk] @ c


def rel(a, b) -> float:
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0))
