"""Test infrastructure only (oracle): restatement of the QRCP point selector.

Follows src/cpu/getpoints_QRCP.cpp:11-500 at one rank:
  * numPre = IRound(sqrt(mu * f)), f = 1.5 in the reference (:82-83); error
    when numPre > nstate (:84-86) or numPre^2 > Ng (:423-427);
  * srand48(seed) (isdf.cpp:68: 41), G1 (K1 x numPre) then G2 (K2 x numPre)
    filled column-major with sqrt(-2 log a) cos(2 pi b), a, b = drand48()
    (include/common/utility.hpp:455-471);
  * Orth = LAPACK dgesvd jobu='O' (src/cpu/lapack.cpp:115-147);
  * psiG1 = psi_S1 G1, phiG2 = psi_S2 G2 (:201-207);
  * MG(i + j*numPre, r) = phiG2(r, i) * psiG1(r, j), squared column norms
    summed j-outer, i-inner (:228-235);
  * keep the columns with norm > 1e-5 * max, ascending (:272-284);
  * column-pivoted QR of the kept columns; the reference calls ScaLAPACK
    pdgeqpf (:440, src/cpu/scalapack.cpp:44-54), which is not available here:
    this restatement calls LAPACK dgeqpf (the same unblocked Householder CPQR
    with norm downdating) from scipy's OpenBLAS, or its C restatement
    (oracle/qrcp_port.cpp: port_dgeqpf), which can stop after a prefix of
    pivots and follow a forced pivot sequence;
  * piv[j] = MGIdx[pivot_j] for j < ntotMG, 0 after (:454-457).
Only tests import this module.
"""
from __future__ import annotations

import ctypes
import glob
import math
import os

import numpy as np
import scipy
import scipy.linalg as sl

PI = 3.14159265358979323846  # include/common/environment.hpp


def iround(a: float) -> int:
    """IRound, include/common/utility.hpp:18-23."""
    if a > 0:
        return int(a) if a - int(a) < 0.5 else int(a) + 1
    return int(a) if int(a) - a < 0.5 else int(a) - 1


def num_pre(mu: int, factor: float = 1.5) -> int:
    return iround(math.sqrt(mu * factor))


_libc = ctypes.CDLL(None)
_libc.drand48.restype = ctypes.c_double
_libc.srand48.argtypes = [ctypes.c_long]


def gaussians(k1: int, k2: int, p: int, seed: int):
    """Raw G1, G2 (before Orth), F-order, drawn as the reference draws them."""
    _libc.srand48(seed)

    def fill(m, n):
        g = np.empty(m * n)
        for e in range(m * n):
            a = _libc.drand48()
            b = _libc.drand48()
            g[e] = math.sqrt(-2.0 * math.log(a)) * math.cos(2.0 * PI * b)
        return g.reshape(n, m).T.copy(order="F")

    g1 = fill(k1, p)
    g2 = fill(k2, p)
    return g1, g2


def orth(g):
    """dgesvd jobu='O': the left singular vectors overwrite G."""
    u, _, _ = sl.svd(g, full_matrices=False, lapack_driver="gesvd")
    return np.asfortranarray(u)


def sketch(k1, k2, p, seed):
    g1, g2 = gaussians(k1, k2, p, seed)
    return orth(g1), orth(g2)


def _openblas():
    d = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
    lib = ctypes.CDLL(glob.glob(os.path.join(d, "libscipy_openblas*.so"))[0])
    lib.scipy_dgeqpf_.restype = None
    return lib


def dgeqpf(a):
    """LAPACK dgeqpf on a copy of a (F-order); returns 0-based pivots and tau."""
    a = np.array(a, dtype=np.float64, order="F", copy=True)
    m, n = a.shape
    jpvt = np.zeros(n, dtype=np.int32)
    tau = np.zeros(min(m, n))
    work = np.zeros(3 * n)
    info = ctypes.c_int(0)
    M, N, LDA = ctypes.c_int(m), ctypes.c_int(n), ctypes.c_int(m)
    P = lambda x: x.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    _openblas().scipy_dgeqpf_(ctypes.byref(M), ctypes.byref(N), P(a), ctypes.byref(LDA), P(jpvt),
                              P(tau), P(work), ctypes.byref(info))
    if info.value != 0:
        raise RuntimeError(f"dgeqpf info={info.value}")
    return jpvt.astype(np.int64) - 1, a


def mg_norms(psig1, phig2):
    """Squared MG column norms, summed in the reference's loop order."""
    p = psig1.shape[1]
    s = np.zeros(psig1.shape[0])
    for j in range(p):
        for i in range(p):
            mg = phig2[:, i] * psig1[:, j]
            s += mg * mg
    return s


def select(psi, nocc, nv1, nc1, nv2, nc2, mu, seed=41, factor=1.5, g=None):
    """Returns (piv int32[Ng], ntotMG, pivots over MGIdx, MGIdx, MG norms)."""
    psi = np.asarray(psi)
    ng, nstate = psi.shape
    p = num_pre(mu, factor)
    if p > nstate:
        raise ValueError("numMu is too large for interpolative separable density fitting!")
    k1, k2 = nv1 + nc1, nv2 + nc2
    g1, g2 = g if g is not None else sketch(k1, k2, p, seed)
    psig1 = psi[:, nocc - nv1:nocc + nc1] @ g1
    phig2 = psi[:, nocc - nv2:nocc + nc2] @ g2
    norms = mg_norms(psig1, phig2)
    mx = norms.max()
    idx = np.nonzero(norms > mx * 1e-5)[0]
    if p * p > ng:
        raise ValueError("numPre*numPre > ntot")
    mg = (phig2[idx][:, None, :] * psig1[idx][:, :, None]).reshape(len(idx), p * p).T
    piv_mg, _ = dgeqpf(mg)
    piv = np.zeros(ng, dtype=np.int32)
    piv[:len(idx)] = idx[piv_mg]
    return piv, len(idx), piv_mg, idx, norms


def residual_norms(mg, selected):
    """Norms of every column of mg after projecting out the selected columns."""
    if len(selected) == 0:
        return np.linalg.norm(mg, axis=0)
    q, _ = np.linalg.qr(mg[:, selected])
    r = mg - q @ (q.T @ mg)
    return np.linalg.norm(r, axis=0)


# ----------------------------------------------------------------- C restatement
def _port():
    from oracle import port

    L = port.lib()
    if not getattr(L, "_qrcp_bound", False):
        P, I, LL = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong
        L.port_qrcp_mg.argtypes = [P, P, LL, I, P, I, P]
        L.port_dgeqpf.argtypes = [P, LL, LL, I, P, P, P, P, P]
        L.port_dgeqpf.restype = LL
        L._qrcp_bound = True
    return L


def _p(x):
    return None if x is None else x.ctypes.data_as(ctypes.c_void_p)


def mg_matrix(A, B, idx):
    """MG restricted to the kept columns idx: p^2 x len(idx), F-order."""
    A = np.asfortranarray(A, dtype=np.float64)
    B = np.asfortranarray(B, dtype=np.float64)
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    p = A.shape[1]
    mg = np.empty((p * p, len(idx)), order="F")
    _port().port_qrcp_mg(_p(A), _p(B), A.shape[0], p, _p(idx), len(idx), _p(mg))
    return mg


def dgeqpf_port(mg, kmax=None, forced=None):
    """port_dgeqpf on mg (overwritten). Returns (order, free_choice, max_norm,
    taken_norm, recomputes): order[i] = the column taken at step i (0-based
    column of mg); free_choice[i] = the column dgeqpf itself picks at step i
    given the columns taken before; max_norm / taken_norm their norms."""
    m, n = mg.shape
    assert mg.flags.f_contiguous and mg.dtype == np.float64
    k = min(m, n) if kmax is None else min(kmax, m, n)
    jpvt = np.zeros(n, dtype=np.int32)
    free = np.zeros(k, dtype=np.int32)
    mx = np.zeros(k)
    tk = np.zeros(k)
    f = None
    if forced is not None:
        f = np.full(k, -1, dtype=np.int32)
        f[:min(k, len(forced))] = np.asarray(forced[:k], dtype=np.int32)
    rec = _port().port_dgeqpf(_p(mg), m, n, k, _p(f), _p(jpvt), _p(free), _p(mx), _p(tk))
    if rec < 0:
        raise ValueError("a forced pivot names a column taken at an earlier step")
    return jpvt[:k].astype(np.int64), free.astype(np.int64), mx, tk, int(rec)


def sketch_operands(psi, nocc, nv1, nc1, nv2, nc2, mu, seed=41, factor=1.5):
    """(A, B, kept columns idx, numPre) of the reference's QRCP selector."""
    psi = np.asarray(psi)
    p = num_pre(mu, factor)
    g1, g2 = sketch(nv1 + nc1, nv2 + nc2, p, seed)
    A = np.asfortranarray(psi[:, nocc - nv1:nocc + nc1] @ g1)
    B = np.asfortranarray(psi[:, nocc - nv2:nocc + nc2] @ g2)
    norms = mg_norms(A, B)
    idx = np.nonzero(norms > norms.max() * 1e-5)[0]
    return A, B, idx, p


def follow_pivots(psi, nocc, nv1, nc1, nv2, nc2, mu, piv_other, seed=41, factor=1.5,
                  kmax=None):
    """Runs the dgeqpf restatement on the reference's MG while taking, at every
    step, the grid point that another implementation picked (piv_other, grid
    indices in pivot order). Returns per step: the grid point dgeqpf would
    have picked, the largest remaining norm, the norm of the point taken, the
    number of steps, the largest column norm and the recompute count."""
    A, B, idx, p = sketch_operands(psi, nocc, nv1, nc1, nv2, nc2, mu, seed, factor)
    k = min(mu, len(idx), p * p) if kmax is None else min(kmax, mu, len(idx), p * p)
    col_of = {int(g): c for c, g in enumerate(idx)}
    forced = np.array([col_of.get(int(g), -2) for g in piv_other[:k]], dtype=np.int64)
    if (forced < 0).any():
        raise ValueError("a pivot of the other run is not a kept MG column")
    mg = mg_matrix(A, B, idx)
    top = float(np.sqrt((mg * mg).sum(axis=0).max()))
    _, free, mx, tk, rec = dgeqpf_port(mg, k, forced)
    return idx[free], mx, tk, k, top, rec

