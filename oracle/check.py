"""Test infrastructure only (oracle): numpy restatement of the ISDF check.

Follows src/common/checkcode.cpp:54-313 at one rank:
  * pair densities rho_ij(r) = psi_k(r) psi_j(r), k in S1 (outer), j in S2,
    column (k - lo1) * n2 + (j - lo2)                      (:62-73)
  * C(mu, ij) = psi(piv_mu, k) psi(piv_mu, j)              (:129-139)
  * fit error ||rho - theta C||_F / ||rho||_F              (:146-166)
  * truncated Coulomb kernel, R = 5: V(G) = 4 pi R^2 at G = 0 (gkk < 1e-8),
    else 8 pi / (2 gkk) (1 - cos(sqrt(2 gkk) R)), gkk = |G|^2 / 2
    (:168-182, src/common/fourier.cpp:55-94)
  * forward FFTs scaled by vol / Ng (fourier.cpp:191-196), full spectrum
  * (ij|V|kl) = Re(rho^H V rho), ISDF form C^T Re(zeta^H V zeta) C, relative
    Frobenius error                                        (:184-312)
numpy's FFT replaces FFTW. Only tests import this module.
"""
from __future__ import annotations

import numpy as np

PI = 3.14159265358979323846


def coulomb_kernel(ng, length, radius=5.0):
    """V on the full FFT grid in numpy's (z, y, x) axis order."""
    ks = []
    for d in range(3):
        n = ng[d]
        k = np.array([i if i <= n // 2 else i - n for i in range(n)], dtype=np.float64)
        ks.append(k * 2.0 * PI / length[d])
    kz, ky, kx = np.meshgrid(ks[2], ks[1], ks[0], indexing="ij")
    gkk = (kx * kx + ky * ky + kz * kz) / 2.0
    with np.errstate(divide="ignore", invalid="ignore"):
        v = 8.0 * PI / (2.0 * gkk) * (1 - np.cos(np.sqrt(2.0 * gkk) * radius))
    v[gkk < 1e-8] = 4.0 * PI * radius * radius
    return v


def _spectra(cols, ng, length):
    nx, ny, nz = ng
    vol = length[0] * length[1] * length[2]
    a = cols.T.reshape(cols.shape[1], nz, ny, nx)
    return np.fft.fftn(a, axes=(1, 2, 3)).reshape(cols.shape[1], -1) * (vol / (nx * ny * nz))


def check(psi, ng, length, nocc, nv1, nc1, nv2, nc2, rk, piv, theta):
    """(fit error, Coulomb error)."""
    psi = np.asarray(psi)
    a = psi[:, nocc - nv1:nocc + nc1]
    b = psi[:, nocc - nv2:nocc + nc2]
    rho = (a[:, :, None] * b[:, None, :]).reshape(psi.shape[0], -1)
    p = np.asarray(piv[:rk], dtype=np.int64)
    c = (a[p][:, :, None] * b[p][:, None, :]).reshape(rk, -1)
    fit = theta[:, :rk] @ c
    fit_err = np.linalg.norm(rho - fit) / np.linalg.norm(rho)
    v = coulomb_kernel(ng, length).reshape(-1)
    r_hat = _spectra(rho, ng, length)
    ijkl = np.real(np.conj(r_hat) @ (v[:, None] * r_hat.T))
    z_hat = _spectra(np.asarray(theta[:, :rk]), ng, length)
    aux = np.real(np.conj(z_hat) @ (v[:, None] * z_hat.T))
    isdf = c.T @ aux @ c
    coul_err = np.linalg.norm(ijkl - isdf) / np.linalg.norm(ijkl)
    return float(fit_err), float(coul_err)


def check_sampled(psi, ng, length, nocc, nv1, nc1, nv2, nc2, rk, piv, theta, pairs,
                  fitted_spectra=False):
    """The check's two errors restricted to the state pairs `pairs` (pair
    index (k - lo1) * n2 + (j - lo2), checkcode.cpp:62-73): the fit error over
    all grid points of those pairs and the relative Coulomb error of the pair
    block (ij|V|kl). fitted_spectra=False evaluates the ISDF form as the
    reference does, c_ij^T Re(zeta^H V zeta) c_kl with zeta the spectra of
    every theta column (checkcode.cpp:249-288); True takes the spectra of the
    fitted densities theta c_ij instead (the same number by linearity of the
    FFT, at 2 len(pairs) transforms: what sizes beyond Si8 need)."""
    psi = np.asarray(psi)
    pairs = np.asarray(pairs, dtype=np.int64)
    n2 = nv2 + nc2
    k = nocc - nv1 + pairs // n2
    j = nocc - nv2 + pairs % n2
    rho = psi[:, k] * psi[:, j]
    p = np.asarray(piv[:rk], dtype=np.int64)
    c = psi[p][:, k] * psi[p][:, j]  # rk x npair_s
    fit = theta[:, :rk] @ c
    fit_err = np.linalg.norm(rho - fit) / np.linalg.norm(rho)
    v = coulomb_kernel(ng, length).reshape(-1)
    r_hat = _spectra(rho, ng, length)
    ijkl = np.real(np.conj(r_hat) @ (v[:, None] * r_hat.T))
    if fitted_spectra:
        f_hat = _spectra(fit, ng, length)
        isdf = np.real(np.conj(f_hat) @ (v[:, None] * f_hat.T))
    else:
        z_hat = _spectra(np.asarray(theta[:, :rk]), ng, length)
        aux = np.real(np.conj(z_hat) @ (v[:, None] * z_hat.T))
        isdf = c.T @ aux @ c
    coul_err = np.linalg.norm(ijkl - isdf) / np.linalg.norm(ijkl)
    return float(fit_err), float(coul_err)


def coulomb_matrix(theta, ng, length, rk):
    """Re(zeta^H V zeta), zeta the full spectra of the theta columns scaled by
    vol/Ng (checkcode.cpp:249-288)."""
    v = coulomb_kernel(ng, length).reshape(-1)
    z_hat = _spectra(np.asarray(theta[:, :rk]), ng, length)
    return np.real(np.conj(z_hat) @ (v[:, None] * z_hat.T))
