"""Test infrastructure only (oracle): ctypes bindings of oracle/_ref/libisdf_ref.so.

That library is the reference's own CPU code for the ISDF path (K-means
selection in src/common/utility.cpp:631-988, the FP64 fit in
src/cpu/getbasis_MPI.cpp, the check in src/common/checkcode.cpp) compiled by
oracle/build_ref.sh with single-rank shims. Only tests, the smoke check and
bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libisdf_ref.so")
LIB_MP_PATH = os.path.join(_HERE, "_ref", "libisdf_ref_mp.so")
_lib = None
_lib_mp = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        I = ctypes.c_int
        _lib.ref_kmeans_piv.argtypes = [P, P, P, I, I, I, I, I, I, I, I, ctypes.c_uint, I, P, P, P,
                                        P, P, I]
        _lib.ref_getbasis.argtypes = [P, P, P, I, I, I, I, I, I, I, P, P, P, I]
        _lib.ref_checkcode.argtypes = [P, P, P, I, I, I, I, I, I, I, P, P, P, P, P, I]
        _lib.ref_weight.argtypes = [P, I, I, I, I, I, I, P]
        _lib.ref_bench_kmeans_step.argtypes = [I, I, I]
        _lib.ref_bench_kmeans_step.restype = ctypes.c_double
        _lib.ref_qrcp_sketch.argtypes = [I, I, I, ctypes.c_long, P, P]
        _lib.ref_qrcp_gaussians.argtypes = [I, I, I, ctypes.c_long, P, P]
        _lib.ref_kmeans_warm.argtypes = [P, P, P, I, I, P, P, P, P, P, I]
        _lib.ref_bench_kmean.argtypes = [P, P, P, I, I, P]
        _lib.ref_bench_kmean.restype = ctypes.c_double
        _lib.ref_iround.argtypes = [ctypes.c_double]
        _lib.ref_iround.restype = I
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _geom(ng, length):
    ng = np.ascontiguousarray(ng, dtype=np.int32)
    ln = np.ascontiguousarray(length, dtype=np.float64)
    return ng, ln


class OracleError(RuntimeError):
    pass


def weight(psi, nocc, nv1, nc1, nv2, nc2):
    psi = np.asfortranarray(psi, dtype=np.float64)
    w = np.empty(psi.shape[0])
    lib().ref_weight(_ptr(psi), psi.shape[0], nocc, nv1, nc1, nv2, nc2, _ptr(w))
    return w


def kmeans_piv(psi, ng, length, nocc, nv1, nc1, nv2, nc2, mu, iters, rand_seed=1,
               cross_check=False):
    """Returns (piv int32[Ng], rk_eff, iterations run, weight)."""
    psi = np.asfortranarray(psi, dtype=np.float64)
    g, ln = _geom(ng, length)
    n = int(np.prod(g))
    assert psi.shape[0] == n
    piv = np.zeros(n, dtype=np.int32)
    rk = np.zeros(1, dtype=np.int32)
    it = np.zeros(1, dtype=np.int32)
    w = np.empty(n)
    log = ctypes.create_string_buffer(1 << 16)
    rc = lib().ref_kmeans_piv(_ptr(psi), _ptr(g), _ptr(ln), nocc, psi.shape[1], nv1, nc1, nv2,
                              nc2, mu, iters, rand_seed, int(cross_check), _ptr(piv), _ptr(rk),
                              _ptr(it), _ptr(w), log, len(log))
    if rc != 0:
        raise OracleError(f"ref_kmeans_piv rc={rc}: {log.value.decode(errors='replace')[-400:]}")
    return piv, int(rk[0]), int(it[0]), w


def kmeans_warm(w, ng, length, mu, iters, prev_piv):
    """The reference's KMEAN on weight w with piv = prev_piv on entry (its warm
    start when prev_piv[0] != prev_piv[1]). Returns (piv, rk_eff, iterations,
    "Reusable pivots" as logged or -1)."""
    w = np.ascontiguousarray(w, dtype=np.float64)
    g, ln = _geom(ng, length)
    piv = np.array(prev_piv, dtype=np.int32, copy=True)
    rk = np.zeros(1, dtype=np.int32)
    it = np.zeros(1, dtype=np.int32)
    used = np.zeros(1, dtype=np.int32)
    log = ctypes.create_string_buffer(1 << 16)
    rc = lib().ref_kmeans_warm(_ptr(w), _ptr(g), _ptr(ln), mu, iters, _ptr(piv), _ptr(rk),
                               _ptr(it), _ptr(used), log, len(log))
    if rc != 0:
        raise OracleError(f"ref_kmeans_warm rc={rc}: {log.value.decode(errors='replace')[-400:]}")
    return piv, int(rk[0]), int(it[0]), int(used[0])


def getbasis(psi, ng, length, nocc, nv1, nc1, nv2, nc2, rk, piv):
    """theta (Ng x rk, F-order) from the reference's getbasis_MPI at one rank."""
    psi = np.asfortranarray(psi, dtype=np.float64)
    g, ln = _geom(ng, length)
    n = int(np.prod(g))
    piv = np.ascontiguousarray(piv, dtype=np.int32)
    theta = np.zeros((n, rk), dtype=np.float64, order="F")
    log = ctypes.create_string_buffer(1 << 14)
    rc = lib().ref_getbasis(_ptr(psi), _ptr(g), _ptr(ln), nocc, psi.shape[1], nv1, nc1, nv2, nc2,
                            rk, _ptr(piv), _ptr(theta), log, len(log))
    if rc != 0:
        raise OracleError(f"ref_getbasis rc={rc}: {log.value.decode(errors='replace')[-400:]}")
    return theta


def checkcode(psi, ng, length, nocc, nv1, nc1, nv2, nc2, rk, piv, theta):
    """(fit error, Coulomb error) as printed by the reference's checkcode."""
    psi = np.asfortranarray(psi, dtype=np.float64)
    theta = np.asfortranarray(theta, dtype=np.float64)
    g, ln = _geom(ng, length)
    piv = np.ascontiguousarray(piv, dtype=np.int32)
    fe = np.zeros(1)
    ce = np.zeros(1)
    log = ctypes.create_string_buffer(1 << 14)
    rc = lib().ref_checkcode(_ptr(psi), _ptr(g), _ptr(ln), nocc, psi.shape[1], nv1, nc1, nv2, nc2,
                             rk, _ptr(piv), _ptr(theta), _ptr(fe), _ptr(ce), log, len(log))
    if rc != 0:
        raise OracleError(f"ref_checkcode rc={rc}: {log.value.decode(errors='replace')[-400:]}")
    return float(fe[0]), float(ce[0])


def iround(a: float) -> int:
    return int(lib().ref_iround(float(a)))


def bench_kmeans_step(npt: int, rk: int, repeats: int = 1) -> float:
    """Seconds of one reference Lloyd step (pdist2 + findMin) at full size."""
    return float(lib().ref_bench_kmeans_step(npt, rk, repeats))


def bench_kmean(w, ng, length, mu: int, iters: int) -> float:
    """Seconds of the reference's whole KMEAN with KmeansMaxIter = iters."""
    w = np.ascontiguousarray(w, dtype=np.float64)
    g, ln = _geom(ng, length)
    piv = np.zeros(w.shape[0], dtype=np.int32)
    return float(lib().ref_bench_kmean(_ptr(w), _ptr(g), _ptr(ln), mu, iters, _ptr(piv)))


def bench_getbasis_rows(psi, shape, fraction: int, repeats: int = 1) -> float:
    """Seconds of the reference's getbasis_MPI on the first Ng/fraction grid
    rows with the full mu (pivots drawn inside that row block)."""
    import time

    rows = psi.shape[0] // fraction
    sub = np.asfortranarray(psi[:rows])
    piv = np.random.default_rng(0).choice(rows, size=shape.mu, replace=False).astype(np.int32)
    piv = np.concatenate([np.sort(piv), np.zeros(rows - shape.mu, dtype=np.int32)])
    best = 1e300
    for _ in range(repeats):
        t0 = time.perf_counter()
        getbasis(sub, (rows, 1, 1), (1.0, 1.0, 1.0), shape.nocc, shape.nv1, shape.nc1, shape.nv2,
                 shape.nc2, shape.mu, piv)
        best = min(best, time.perf_counter() - t0)
    return best


def qrcp_sketch(k1: int, k2: int, num_pre: int, seed: int, orth: bool = True):
    """G1, G2 of the reference's QRCP (srand48 + GaussianRandom [+ lapack::Orth])."""
    g1 = np.zeros((k1, num_pre), order="F")
    g2 = np.zeros((k2, num_pre), order="F")
    f = lib().ref_qrcp_sketch if orth else lib().ref_qrcp_gaussians
    f(k1, k2, num_pre, seed, _ptr(g1), _ptr(g2))
    return g1, g2


def available_ranks() -> bool:
    return os.path.exists(LIB_MP_PATH)


def kmeans_ranks(w, ng, length, mu, iters, ranks, rand_seed=1, timeout_s=600.0):
    """The reference's own KMEAN (src/common/utility.cpp:631-988) run as
    `ranks` MPI ranks: forked processes over the shared-memory MPI stand-in of
    oracle/shims_mp (reductions in binomial-tree order). Tolerances of the GPU
    path (1e-5, 1e-8), piv zeroed first. Returns (piv, rk_eff, iterations)."""
    global _lib_mp
    if _lib_mp is None:
        _lib_mp = ctypes.CDLL(LIB_MP_PATH)
        P, I = ctypes.c_void_p, ctypes.c_int
        _lib_mp.ref_kmeans_ranks.argtypes = [I, P, P, P, I, I, I, ctypes.c_uint, P, P, P,
                                             ctypes.c_double]
        _lib_mp.ref_kmeans_ranks.restype = I
    w = np.ascontiguousarray(w, dtype=np.float64)
    g, ln = _geom(ng, length)
    piv = np.zeros(w.shape[0], dtype=np.int32)
    rk = np.zeros(1, dtype=np.int32)
    it = np.zeros(1, dtype=np.int32)
    rc = _lib_mp.ref_kmeans_ranks(ranks, _ptr(w), _ptr(g), _ptr(ln), mu, iters, 0, rand_seed,
                                  _ptr(piv), _ptr(rk), _ptr(it), float(timeout_s))
    if rc != 0:
        raise OracleError(f"ref_kmeans_ranks({ranks}) failed: {rc}")
    return piv, int(rk[0]), int(it[0])
