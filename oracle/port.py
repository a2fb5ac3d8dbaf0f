"""Test infrastructure only (oracle): bindings of the CPU restatements.

libisdf_port.so (oracle/kmeans_port.cpp) restates the reference's weight and
K-means selection bit for bit; fit.py restates the FP64 fit. Only tests, the
smoke check and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libisdf_port.so")
_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(LIB_PATH)
        P, I = ctypes.c_void_p, ctypes.c_int
        _lib.port_weight.argtypes = [P, ctypes.c_longlong, I, I, I, I, I, P]
        _lib.port_kmeans.argtypes = [P, I, P, P, I, I, ctypes.c_longlong, P, P]
        _lib.port_kmeans.restype = I
        _lib.port_kmeans_warm.argtypes = [P, I, P, P, I, I, ctypes.c_longlong, P, P, I, P]
        _lib.port_kmeans_warm.restype = I
        _lib.port_kmeans_ranks.argtypes = [P, I, P, P, I, I, ctypes.c_longlong, P, P, I, P, I]
        _lib.port_kmeans_ranks.restype = I
        _lib.port_num_threads.restype = I
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def weight(psi, nocc, nv1, nc1, nv2, nc2):
    psi = np.asfortranarray(psi, dtype=np.float64)
    w = np.empty(psi.shape[0])
    lib().port_weight(_ptr(psi), psi.shape[0], nocc, nv1, nc1, nv2, nc2, _ptr(w))
    return w


def kmeans(w, ng, length, mu, iters, rand_seed=1):
    """Returns (piv int32[Ng], rk_eff, iterations run)."""
    w = np.ascontiguousarray(w, dtype=np.float64)
    g = np.ascontiguousarray(ng, dtype=np.int32)
    ln = np.ascontiguousarray(length, dtype=np.float64)
    piv = np.zeros(w.shape[0], dtype=np.int32)
    it = np.zeros(1, dtype=np.int32)
    rk = lib().port_kmeans(_ptr(w), w.shape[0], _ptr(g), _ptr(ln), mu, iters, rand_seed, _ptr(piv),
                           _ptr(it))
    if rk <= 0:
        raise RuntimeError(f"port_kmeans failed: {rk}")
    return piv, rk, int(it[0])


def kmeans_warm(w, ng, length, mu, iters, prev_piv, rand_seed=1):
    """K-means started from the previous pivots prev_piv (used when
    prev_piv[0] != prev_piv[1], utility.cpp:725-749). Returns (piv, rk_eff,
    iterations run, previous pivots kept as initial centroids or -1)."""
    w = np.ascontiguousarray(w, dtype=np.float64)
    g = np.ascontiguousarray(ng, dtype=np.int32)
    ln = np.ascontiguousarray(length, dtype=np.float64)
    piv = np.array(prev_piv, dtype=np.int32, copy=True)
    assert piv.size == w.shape[0]
    it = np.zeros(1, dtype=np.int32)
    used = np.zeros(1, dtype=np.int32)
    rk = lib().port_kmeans_warm(_ptr(w), w.shape[0], _ptr(g), _ptr(ln), mu, iters, rand_seed,
                                _ptr(piv), _ptr(it), 1, _ptr(used))
    if rk <= 0:
        raise RuntimeError(f"port_kmeans_warm failed: {rk}")
    return piv, rk, int(it[0]), int(used[0])


def kmeans_ranks(w, ng, length, mu, iters, ranks, rand_seed=1):
    """K-means as `ranks` MPI ranks would run the reference's KMEAN (the point
    partition, per-rank sums combined in binomial-tree order, MINLOC for the
    nearest points; oracle/kmeans_port.cpp). Returns (piv, rk_eff, iterations)."""
    w = np.ascontiguousarray(w, dtype=np.float64)
    g = np.ascontiguousarray(ng, dtype=np.int32)
    ln = np.ascontiguousarray(length, dtype=np.float64)
    piv = np.zeros(w.shape[0], dtype=np.int32)
    it = np.zeros(1, dtype=np.int32)
    rk = lib().port_kmeans_ranks(_ptr(w), w.shape[0], _ptr(g), _ptr(ln), mu, iters, rand_seed,
                                 _ptr(piv), _ptr(it), 0, None, ranks)
    if rk <= 0:
        raise RuntimeError(f"port_kmeans_ranks failed: {rk}")
    return piv, rk, int(it[0])


def kmeans_piv(psi, ng, length, nocc, nv1, nc1, nv2, nc2, mu, iters, rand_seed=1):
    w = weight(psi, nocc, nv1, nc1, nv2, nc2)
    piv, rk, it = kmeans(w, ng, length, mu, iters, rand_seed)
    return piv, rk, it, w


def num_threads() -> int:
    return int(lib().port_num_threads())
