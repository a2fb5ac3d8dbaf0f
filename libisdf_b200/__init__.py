"""libisdf_b200: a B200-native ISDF engine behind LibISDF's GPU ISDF() interface.

The compute path is libisdf_b200.so (hand-written sm_100a CUDA kernels behind
the C ABI in include/isdf_c.h). This module binds that ABI with ctypes and
mirrors the reference's entry point

    isdf::isdffunc::ISDF(d_psirow, domain, nocc, nstate, nv1, nc1, nv2, nc2,
                         mu_points, d_thetaCol, piv, KmeansMaxIter_ISDF, check)

(reference include/isdf.hpp:37, src/common/isdf.cpp:132-209) with the
Kmeans/QRCP selector of its CPU overload (isdf.hpp:39). Device buffers are
torch CUDA tensors (float64, column-major data: a tensor of shape
(nstate, Ng) row-major is the same bytes as Ng x nstate column-major) or raw
device pointers; piv is a host int32 numpy array of length Ng.

There is no CPU fallback: if the shared library is missing, importing the
binding raises.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libisdf_b200.so")

ISDF_OK = 0
ISDF_ERR_ARG = -1
ISDF_ERR_CUDA = -2
ISDF_ERR_NOMEM = -3
ISDF_ERR_NOT_SPD = -4
ISDF_ERR_TIMEOUT = -5
ISDF_ERR_UNSUPPORTED = -6
ISDF_ERR_CANCELLED = -7
ISDF_ERR_BUSY = -8
ISDF_ERR_COMM = -9

SELECT_KMEANS = 0
SELECT_QRCP = 1
PRECISION_FP64 = 0
PRECISION_MIXED = 1
THETA_ROWS = 0
THETA_CYCLIC = 1


class IsdfError(RuntimeError):
    """Raised for a non-zero status (the reference throws std::runtime_error)."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


class _Domain(ctypes.Structure):
    _fields_ = [("length", ctypes.c_double * 3), ("pos_start", ctypes.c_double * 3),
                ("num_grid", ctypes.c_int * 3), ("num_grid_fine", ctypes.c_int * 3)]


class _Options(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("refine_steps", ctypes.c_int),
                ("qrcp_oversample", ctypes.c_double), ("qrcp_seed", ctypes.c_longlong),
                ("rand_seed", ctypes.c_longlong), ("stream", ctypes.c_void_p),
                ("mixed_slices", ctypes.c_int), ("kmeans_warm_start", ctypes.c_int),
                ("reserved", ctypes.c_int * 6)]


class _Report(ctypes.Structure):
    _fields_ = [("rk_requested", ctypes.c_int), ("rk_eff", ctypes.c_int),
                ("kmeans_iters", ctypes.c_int), ("npt", ctypes.c_int),
                ("fit_err", ctypes.c_double), ("coul_err", ctypes.c_double),
                ("t_select_ms", ctypes.c_double), ("t_fit_ms", ctypes.c_double),
                ("t_zct_ms", ctypes.c_double), ("t_chol_ms", ctypes.c_double),
                ("t_solve_ms", ctypes.c_double), ("t_check_ms", ctypes.c_double),
                ("t_total_ms", ctypes.c_double), ("chol_info", ctypes.c_int),
                ("kernel_launches", ctypes.c_int), ("t_gemm_ms", ctypes.c_float),
                ("kmeans_search_frac", ctypes.c_float), ("qrcp_steps", ctypes.c_int),
                ("qrcp_norm_recomputes", ctypes.c_int), ("kmeans_warm_pivots", ctypes.c_int),
                ("reserved", ctypes.c_int * 1)]


class _ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("slots", ctypes.c_int),
                ("hbm_budget_bytes", ctypes.c_size_t), ("max_queue", ctypes.c_int),
                ("max_skips", ctypes.c_int), ("batch_small", ctypes.c_int),
                ("reserved", ctypes.c_int * 3)]


class _Request(ctypes.Structure):
    _fields_ = [("dom", _Domain), ("d_psi", ctypes.c_void_p), ("nocc", ctypes.c_int),
                ("nstate", ctypes.c_int), ("nv1", ctypes.c_int), ("nc1", ctypes.c_int),
                ("nv2", ctypes.c_int), ("nc2", ctypes.c_int), ("mu_points", ctypes.c_int),
                ("d_theta", ctypes.c_void_p), ("piv", ctypes.c_void_p),
                ("kmeans_max_iter", ctypes.c_int), ("selector", ctypes.c_int),
                ("check", ctypes.c_int), ("opt", _Options)]


class _ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_longlong), ("completed", ctypes.c_longlong),
                ("failed", ctypes.c_longlong), ("cancelled", ctypes.c_longlong),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double),
                ("mean_ms", ctypes.c_double), ("solves_per_s", ctypes.c_double),
                ("peak_concurrency", ctypes.c_int), ("queued", ctypes.c_int),
                ("running", ctypes.c_int), ("reserved0", ctypes.c_int),
                ("peak_bytes", ctypes.c_size_t)]


@dataclass
class Domain:
    """Numeric fields of the reference's Domain (include/common/domain.hpp:8-36)."""

    length: tuple
    num_grid: tuple
    pos_start: tuple = (0.0, 0.0, 0.0)
    num_grid_fine: tuple | None = None

    def NumGridTotal(self) -> int:
        return int(self.num_grid[0] * self.num_grid[1] * self.num_grid[2])

    def _c(self) -> _Domain:
        d = _Domain()
        for i in range(3):
            d.length[i] = float(self.length[i])
            d.pos_start[i] = float(self.pos_start[i])
            d.num_grid[i] = int(self.num_grid[i])
            d.num_grid_fine[i] = int((self.num_grid_fine or self.num_grid)[i])
        return d


@dataclass
class Options:
    precision: int = PRECISION_FP64
    refine_steps: int = 0  # FP64 refinement is not built: nonzero is rejected
    qrcp_oversample: float = 1.5
    qrcp_seed: int = 41
    rand_seed: int = -1
    stream: int = 0
    mixed_slices: int = 6
    kmeans_warm_start: bool = False  # reuse the caller's previous piv (utility.cpp:725-749)

    def _c(self) -> _Options:
        o = _Options()
        o.precision = self.precision
        o.refine_steps = self.refine_steps
        o.qrcp_oversample = self.qrcp_oversample
        o.qrcp_seed = self.qrcp_seed
        o.rand_seed = self.rand_seed
        o.stream = self.stream or None
        o.mixed_slices = self.mixed_slices
        o.kmeans_warm_start = int(bool(self.kmeans_warm_start))
        return o


@dataclass
class Report:
    rk_requested: int
    rk_eff: int
    kmeans_iters: int
    npt: int
    fit_err: float
    coul_err: float
    t_select_ms: float
    t_fit_ms: float
    t_zct_ms: float
    t_chol_ms: float
    t_solve_ms: float
    t_check_ms: float
    t_total_ms: float
    chol_info: int
    kernel_launches: int
    t_gemm_ms: float = 0.0
    kmeans_search_frac: float = 0.0
    qrcp_steps: int = 0
    qrcp_norm_recomputes: int = 0
    kmeans_warm_pivots: int = -1


_lib = None


def lib() -> ctypes.CDLL:
    """The loaded libisdf_b200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m libisdf_b200.build` "
                              "(there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        P, I, LL = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong
        L.isdf_solve.argtypes = [ctypes.POINTER(_Domain), P, I, I, I, I, I, I, I, P, P, I, I, I,
                                 ctypes.POINTER(_Options), ctypes.POINTER(_Report)]
        L.isdf_solve.restype = I
        L.isdf_kmeans_weight.argtypes = [P, LL, I, I, I, I, I, I, P, P]
        L.isdf_kmeans_weight.restype = I
        L.isdf_kmeans_select.argtypes = [ctypes.POINTER(_Domain), P, I, I, LL, P, P, P, P, P]
        L.isdf_kmeans_select.restype = I
        L.isdf_kmeans_select_batch.argtypes = [I, P, P, P, P, LL, P, P, P, P, P]
        L.isdf_kmeans_select_batch.restype = I
        L.isdf_fit.argtypes = [P, LL, I, I, I, I, I, I, I, P, P, I, I, P, P]
        L.isdf_fit.restype = I
        L.isdf_check.argtypes = [ctypes.POINTER(_Domain), P, I, I, I, I, I, I, I, P, P, P, P, P]
        L.isdf_check.restype = I
        L.isdf_check_sampled.argtypes = [ctypes.POINTER(_Domain), P, I, I, I, I, I, I, I, P, P, I,
                                         P, P, P, P]
        L.isdf_check_sampled.restype = I
        L.isdf_coulomb_matrix.argtypes = [ctypes.POINTER(_Domain), P, I, P, P]
        L.isdf_coulomb_matrix.restype = I
        L.isdf_last_error.restype = ctypes.c_char_p
        L.isdf_status_string.argtypes = [I]
        L.isdf_status_string.restype = ctypes.c_char_p
        L.isdf_workspace_bytes.argtypes = [LL, I, I, I, I, I]
        L.isdf_workspace_bytes.restype = ctypes.c_size_t
        L.isdf_request_workspace_bytes.argtypes = [ctypes.POINTER(_Domain), I, I, I, I, I, I, I,
                                                   I, ctypes.POINTER(_Options)]
        L.isdf_request_workspace_bytes.restype = ctypes.c_size_t
        L.isdf_default_options.argtypes = [ctypes.POINTER(_Options)]
        L.isdf_comm_nccl_unique_id.argtypes = [P]
        L.isdf_comm_nccl_unique_id.restype = I
        L.isdf_comm_create_nccl.argtypes = [P, I, I, ctypes.POINTER(P)]
        L.isdf_comm_create_nccl.restype = I
        L.isdf_comm_create_local.argtypes = [I, P, ctypes.c_double, P]
        L.isdf_comm_create_local.restype = I
        L.isdf_comm_create_callbacks.argtypes = [P, P, I, I, ctypes.POINTER(P)]
        L.isdf_comm_create_callbacks.restype = I
        L.isdf_comm_rank.argtypes = [P, ctypes.POINTER(I), ctypes.POINTER(I)]
        L.isdf_comm_rank.restype = I
        L.isdf_comm_abort.argtypes = [P]
        L.isdf_comm_abort.restype = I
        L.isdf_comm_destroy.argtypes = [P]
        L.isdf_comm_destroy.restype = I
        L.isdf_row_block.argtypes = [LL, I, I, ctypes.POINTER(LL), ctypes.POINTER(LL)]
        L.isdf_row_block.restype = I
        L.isdf_solve_sharded.argtypes = [P, ctypes.POINTER(_Domain), P, I, I, I, I, I, I, I, P, I,
                                         P, I, ctypes.POINTER(_Options), ctypes.POINTER(_Report)]
        L.isdf_solve_sharded.restype = I
        L.isdf_kmeans_select_sharded.argtypes = [P, ctypes.POINTER(_Domain), P, I, I, LL, P, P,
                                                 P, P]
        L.isdf_kmeans_select_sharded.restype = I
        _lib = L
    return _lib


def _check(rc: int):
    if rc != ISDF_OK:
        msg = lib().isdf_last_error().decode(errors="replace")
        raise IsdfError(rc, msg or lib().isdf_status_string(rc).decode())


def _dptr(x) -> int:
    """Device address of a torch CUDA tensor (or an int address)."""
    if isinstance(x, int):
        return x
    if not getattr(x, "is_cuda", False):
        raise TypeError("expected a CUDA tensor or a device address")
    return int(x.data_ptr())


def _host_int32(piv, n: int) -> np.ndarray:
    if not isinstance(piv, np.ndarray) or piv.dtype != np.int32 or not piv.flags.c_contiguous:
        raise TypeError("piv must be a C-contiguous numpy int32 array (host memory)")
    if piv.size < n:
        raise ValueError(f"piv holds {piv.size} entries, needs {n}")
    return piv


def ISDF(d_psirow, domain: Domain, nocc: int, nstate: int, nv1: int, nc1: int, nv2: int,
         nc2: int, mu_points: int, d_thetaCol, piv: np.ndarray, KmeansMaxIter_ISDF: int,
         s1: str = "Kmeans", check: bool = False, options: Options | None = None) -> Report:
    """The reference's GPU ISDF() (src/common/isdf.cpp:132-209) on one B200.

    Writes theta (Ng x mu, column-major) into d_thetaCol and the pivots into
    the host array piv; raises IsdfError where the reference would throw."""
    sel = {"Kmeans": SELECT_KMEANS, "QRCP": SELECT_QRCP}.get(s1)
    if sel is None:
        raise IsdfError(ISDF_ERR_ARG, "Wrong select points method")
    n = domain.NumGridTotal()
    piv = _host_int32(piv, n)
    d = domain._c()
    o = (options or Options())._c()
    r = _Report()
    rc = lib().isdf_solve(ctypes.byref(d), _dptr(d_psirow), nocc, nstate, nv1, nc1, nv2, nc2,
                          mu_points, _dptr(d_thetaCol), piv.ctypes.data, KmeansMaxIter_ISDF, sel,
                          int(bool(check)), ctypes.byref(o), ctypes.byref(r))
    _check(rc)
    return _report(r)


def kmeans_weight(d_psi, ng: int, nstate: int, nocc: int, nv1: int, nc1: int, nv2: int, nc2: int,
                  d_w, stream: int = 0):
    _check(lib().isdf_kmeans_weight(_dptr(d_psi), ng, nstate, nocc, nv1, nc1, nv2, nc2,
                                    _dptr(d_w), stream or None))


def kmeans_select(domain: Domain, d_w, mu: int, max_iter: int, rand_seed: int = -1,
                  stream: int = 0):
    """Returns (piv int32[Ng], rk_eff, iterations, npt)."""
    n = domain.NumGridTotal()
    piv = np.zeros(n, dtype=np.int32)
    out = (ctypes.c_int * 3)()
    d = domain._c()
    _check(lib().isdf_kmeans_select(ctypes.byref(d), _dptr(d_w), mu, max_iter, rand_seed,
                                    piv.ctypes.data, ctypes.addressof(out),
                                    ctypes.addressof(out) + 4, ctypes.addressof(out) + 8,
                                    stream or None))
    return piv, out[0], out[1], out[2]


def kmeans_select_batch(domains, d_ws, mus, max_iters, rand_seed: int = -1, stream: int = 0):
    """The K-means selections of several small systems in one launch; returns
    a list of (piv int32[Ng], rk_eff, iterations, npt), one per system."""
    n = len(domains)
    doms = (_Domain * n)(*[d._c() for d in domains])
    w = (ctypes.c_void_p * n)(*[_dptr(x) for x in d_ws])
    mu = (ctypes.c_int * n)(*mus)
    it = (ctypes.c_int * n)(*max_iters)
    pivs = [np.zeros(d.NumGridTotal(), dtype=np.int32) for d in domains]
    pp = (ctypes.c_void_p * n)(*[p.ctypes.data for p in pivs])
    rk, its, npt = (ctypes.c_int * n)(), (ctypes.c_int * n)(), (ctypes.c_int * n)()
    _check(lib().isdf_kmeans_select_batch(n, doms, w, mu, it, rand_seed, pp, rk, its, npt,
                                          stream or None))
    return [(pivs[r], rk[r], its[r], npt[r]) for r in range(n)]


def fit(d_psi, ng: int, nstate: int, nocc: int, nv1: int, nc1: int, nv2: int, nc2: int, rk: int,
        piv: np.ndarray, d_theta, precision: int = PRECISION_FP64, refine_steps: int = 0,
        stream: int = 0) -> int:
    """theta for given pivots; returns the Cholesky info (0 = ok)."""
    piv = np.ascontiguousarray(piv, dtype=np.int32)
    info = ctypes.c_int(0)
    rc = lib().isdf_fit(_dptr(d_psi), ng, nstate, nocc, nv1, nc1, nv2, nc2, rk, piv.ctypes.data,
                        _dptr(d_theta), precision, refine_steps, ctypes.addressof(info),
                        stream or None)
    _check(rc)
    return info.value


def check(domain: Domain, d_psi, nocc: int, nstate: int, nv1: int, nc1: int, nv2: int, nc2: int,
          rk: int, piv: np.ndarray, d_theta, stream: int = 0):
    """(fit error, Coulomb error) of theta, as the reference's checkcode computes them."""
    piv = np.ascontiguousarray(piv, dtype=np.int32)
    fe = ctypes.c_double(0.0)
    ce = ctypes.c_double(0.0)
    d = domain._c()
    _check(lib().isdf_check(ctypes.byref(d), _dptr(d_psi), nocc, nstate, nv1, nc1, nv2, nc2, rk,
                            piv.ctypes.data, _dptr(d_theta), ctypes.addressof(fe),
                            ctypes.addressof(ce), stream or None))
    return fe.value, ce.value


def check_sampled(domain: Domain, d_psi, nocc: int, nstate: int, nv1: int, nc1: int, nv2: int,
                  nc2: int, rk: int, piv: np.ndarray, d_theta, pairs, stream: int = 0):
    """(fit error, Coulomb error) of theta restricted to the listed state pairs
    (pair index (k - (nocc-nv1)) * (nv2+nc2) + (j - (nocc-nv2))): the check at
    sizes where all pairs are out of reach. No counterpart in the reference."""
    piv = np.ascontiguousarray(piv, dtype=np.int32)
    pairs = np.ascontiguousarray(pairs, dtype=np.int32)
    fe = ctypes.c_double(0.0)
    ce = ctypes.c_double(0.0)
    d = domain._c()
    _check(lib().isdf_check_sampled(ctypes.byref(d), _dptr(d_psi), nocc, nstate, nv1, nc1, nv2,
                                    nc2, rk, piv.ctypes.data, _dptr(d_theta), len(pairs),
                                    pairs.ctypes.data, ctypes.addressof(fe),
                                    ctypes.addressof(ce), stream or None))
    return fe.value, ce.value


def coulomb_matrix(domain: Domain, d_theta, rk: int, d_A, stream: int = 0):
    """The ISDF Coulomb matrix Re(zeta^H V zeta) (rk x rk) into d_A (device,
    column-major), zeta the spectra of the theta columns (checkcode.cpp:249-288)."""
    d = domain._c()
    _check(lib().isdf_coulomb_matrix(ctypes.byref(d), _dptr(d_theta), rk, _dptr(d_A),
                                     stream or None))


def _report(r: _Report) -> Report:
    return Report(r.rk_requested, r.rk_eff, r.kmeans_iters, r.npt, r.fit_err, r.coul_err,
                  r.t_select_ms, r.t_fit_ms, r.t_zct_ms, r.t_chol_ms, r.t_solve_ms, r.t_check_ms,
                  r.t_total_ms, r.chol_info, r.kernel_launches, r.t_gemm_ms,
                  r.kmeans_search_frac, r.qrcp_steps, r.qrcp_norm_recomputes,
                  r.kmeans_warm_pivots)


class Server:
    """Continuous-batching ISDF server (isdf_server_* C ABI). Requests keep
    references to the caller's buffers (psi, theta on the device, piv on the
    host) until they are done."""

    def __init__(self, slots: int = 4, hbm_budget_bytes: int = 0, device: int = 0,
                 max_skips: int = 64, max_queue: int = 4096, batch_small: int = 32):
        L = lib()
        P, I, LL = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong
        L.isdf_server_create.argtypes = [ctypes.POINTER(_ServerConfig), ctypes.POINTER(P)]
        L.isdf_server_submit.argtypes = [P, ctypes.POINTER(_Request), ctypes.POINTER(LL)]
        L.isdf_server_wait.argtypes = [P, LL, ctypes.c_double, ctypes.POINTER(I),
                                       ctypes.POINTER(_Report)]
        L.isdf_server_poll.argtypes = [P, LL, ctypes.POINTER(I), ctypes.POINTER(I),
                                       ctypes.POINTER(_Report)]
        L.isdf_server_cancel.argtypes = [P, LL]
        L.isdf_server_stats.argtypes = [P, ctypes.POINTER(_ServerStats)]
        L.isdf_server_destroy.argtypes = [P]
        cfg = _ServerConfig()
        cfg.device, cfg.slots, cfg.hbm_budget_bytes = device, slots, hbm_budget_bytes
        cfg.max_queue, cfg.max_skips = max_queue, max_skips
        cfg.batch_small = batch_small
        self._h = ctypes.c_void_p()
        _check(L.isdf_server_create(ctypes.byref(cfg), ctypes.byref(self._h)))
        self._keep = {}

    def submit(self, d_psirow, domain: Domain, nocc, nstate, nv1, nc1, nv2, nc2, mu_points,
               d_thetaCol, piv: np.ndarray, KmeansMaxIter_ISDF: int, s1: str = "Kmeans",
               check: bool = False, options: Options | None = None) -> int:
        n = domain.NumGridTotal()
        piv = _host_int32(piv, n)
        r = _Request()
        r.dom = domain._c()
        r.d_psi = _dptr(d_psirow)
        r.nocc, r.nstate, r.nv1, r.nc1, r.nv2, r.nc2 = nocc, nstate, nv1, nc1, nv2, nc2
        r.mu_points = mu_points
        r.d_theta = _dptr(d_thetaCol)
        r.piv = piv.ctypes.data
        r.kmeans_max_iter = KmeansMaxIter_ISDF
        r.selector = {"Kmeans": SELECT_KMEANS, "QRCP": SELECT_QRCP}[s1]
        r.check = int(bool(check))
        r.opt = (options or Options())._c()
        t = ctypes.c_longlong(0)
        _check(lib().isdf_server_submit(self._h, ctypes.byref(r), ctypes.byref(t)))
        self._keep[t.value] = (d_psirow, d_thetaCol, piv)
        return t.value

    def wait(self, ticket: int, timeout_ms: float = -1.0):
        """(status, Report) once the request is done."""
        st = ctypes.c_int(0)
        rep = _Report()
        _check(lib().isdf_server_wait(self._h, ticket, timeout_ms, ctypes.byref(st),
                                      ctypes.byref(rep)))
        self._keep.pop(ticket, None)
        return st.value, _report(rep)

    def poll(self, ticket: int):
        state, st = ctypes.c_int(0), ctypes.c_int(0)
        rep = _Report()
        _check(lib().isdf_server_poll(self._h, ticket, ctypes.byref(state), ctypes.byref(st),
                                      ctypes.byref(rep)))
        return state.value, st.value

    def cancel(self, ticket: int):
        _check(lib().isdf_server_cancel(self._h, ticket))

    def stats(self) -> dict:
        s = _ServerStats()
        _check(lib().isdf_server_stats(self._h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in _ServerStats._fields_ if k != "reserved0"}

    def close(self):
        if self._h:
            lib().isdf_server_destroy(self._h)
            self._h = ctypes.c_void_p()
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def workspace_bytes(ng: int, nstate: int, mu: int, selector: int = SELECT_KMEANS,
                    precision: int = PRECISION_FP64, check: bool = False) -> int:
    """Footprint at the default QRCP oversampling, without the check's buffers."""
    return int(lib().isdf_workspace_bytes(ng, nstate, mu, selector, precision, int(check)))


def request_workspace_bytes(domain: Domain, nstate: int, nv1: int, nc1: int, nv2: int, nc2: int,
                            mu_points: int, s1: str = "Kmeans", check: bool = False,
                            options: Options | None = None) -> int:
    """The full device footprint of one ISDF() call beyond psi and theta."""
    d = domain._c()
    o = (options or Options())._c()
    sel = {"Kmeans": SELECT_KMEANS, "QRCP": SELECT_QRCP}[s1]
    return int(lib().isdf_request_workspace_bytes(ctypes.byref(d), nstate, nv1, nc1, nv2, nc2,
                                                  mu_points, sel, int(bool(check)),
                                                  ctypes.byref(o)))


# ------------------------------------------------------------------ sharded
def row_block(n: int, size: int, rank: int):
    """(start, count) of rank's block of n grid rows: the reference's rule
    (src/common/isdf.cpp:137-141), the first n % size ranks one row more."""
    a, b = ctypes.c_longlong(), ctypes.c_longlong()
    _check(lib().isdf_row_block(n, size, rank, ctypes.byref(a), ctypes.byref(b)))
    return a.value, b.value


def nccl_unique_id() -> bytes:
    """A new NCCL unique id (128 bytes) for Comm.nccl (NCCL opened at run time)."""
    buf = ctypes.create_string_buffer(128)
    _check(lib().isdf_comm_nccl_unique_id(buf))
    return buf.raw


def share_nccl_unique_id(group=None) -> bytes:
    """A new NCCL unique id made on the group's first rank and handed to every
    rank of a torch.distributed group (broadcast_object_list: any backend,
    gloo included)."""
    import torch.distributed as dist
    box = [nccl_unique_id() if dist.get_rank(group) == 0 else None]
    src = 0 if group is None else dist.get_global_rank(group, 0)
    dist.broadcast_object_list(box, src=src, group=group)
    return box[0]


_SizeP = ctypes.POINTER(ctypes.c_size_t)
_AllgathervFn = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                 ctypes.c_void_p, _SizeP, _SizeP, ctypes.c_void_p)
_AlltoallvFn = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, _SizeP, _SizeP,
                                ctypes.c_void_p, _SizeP, _SizeP, ctypes.c_void_p)


class _CommOps(ctypes.Structure):  # isdf_comm_ops_t
    _fields_ = [("allgatherv", _AllgathervFn), ("alltoallv", _AlltoallvFn)]


class Comm:
    """A rank's communicator for the sharded solve (isdf_comm_t)."""

    def __init__(self, handle: int):
        self._h = ctypes.c_void_p(handle)
        r, n = ctypes.c_int(), ctypes.c_int()
        _check(lib().isdf_comm_rank(self._h, ctypes.byref(r), ctypes.byref(n)))
        self.rank, self.size = r.value, n.value

    @classmethod
    def nccl(cls, unique_id: bytes, rank: int, size: int) -> "Comm":
        """NCCL transport; the current CUDA device is this rank's GPU."""
        if len(unique_id) != 128:
            raise ValueError("an NCCL unique id has 128 bytes")
        h = ctypes.c_void_p()
        _check(lib().isdf_comm_create_nccl(ctypes.create_string_buffer(unique_id, 128), rank,
                                           size, ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def nccl_from_torch(cls, group=None) -> "Comm":
        """NCCL transport for the ranks of a torch.distributed group (any
        backend carries the unique id, see share_nccl_unique_id); the current
        CUDA device is this rank's GPU."""
        import torch.distributed as dist
        uid = share_nccl_unique_id(group)
        return cls.nccl(uid, dist.get_rank(group), dist.get_world_size(group))

    @classmethod
    def local_group(cls, size: int, devices=None, timeout_s: float = 60.0) -> list:
        """`size` ranks inside this process (one host thread per rank calls the
        sharded functions); devices: rank r's GPU (None: all on the current
        device)."""
        hs = (ctypes.c_void_p * size)()
        dv = (ctypes.c_int * size)(*devices) if devices is not None else None
        _check(lib().isdf_comm_create_local(size, dv, float(timeout_s), hs))
        return [cls(hs[r]) for r in range(size)]

    @classmethod
    def callbacks(cls, allgatherv, alltoallv, rank: int, size: int) -> "Comm":
        """Transport over the caller's own collectives (isdf_comm_create_callbacks):
        allgatherv(d_send, send_bytes, d_recv, recv_bytes, recv_displs, stream)
        and alltoallv(d_send, send_bytes, send_displs, d_recv, recv_bytes,
        recv_displs, stream) get device addresses and the cudaStream_t as ints
        and the per-rank byte counts and displacements as lists. The data must
        have arrived, or be ordered on the stream, when they return; an
        exception fails the collective (ISDF_ERR_COMM)."""
        def lst(ptr):
            return [int(ptr[q]) for q in range(size)]

        def agv(ctx, d_send, send_bytes, d_recv, counts, displs, stream):
            try:
                allgatherv(d_send or 0, int(send_bytes), d_recv or 0, lst(counts), lst(displs),
                           stream or 0)
                return 0
            except Exception:  # noqa: BLE001 - reported to the library as a failure
                return 1

        def a2a(ctx, d_send, scounts, sdispls, d_recv, rcounts, rdispls, stream):
            try:
                alltoallv(d_send or 0, lst(scounts), lst(sdispls), d_recv or 0, lst(rcounts),
                          lst(rdispls), stream or 0)
                return 0
            except Exception:  # noqa: BLE001 - reported to the library as a failure
                return 1

        fns = (_AllgathervFn(agv), _AlltoallvFn(a2a))
        ops = _CommOps(*fns)
        h = ctypes.c_void_p()
        _check(lib().isdf_comm_create_callbacks(ctypes.byref(ops), None, rank, size,
                                                ctypes.byref(h)))
        c = cls(h.value)
        c._callbacks = fns  # the library calls these for the communicator's lifetime
        return c

    def abort(self):
        _check(lib().isdf_comm_abort(self._h))

    def close(self):
        if self._h:
            lib().isdf_comm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_sharded(comm: Comm, d_psirow, domain: Domain, nocc: int, nstate: int, nv1: int,
                  nc1: int, nv2: int, nc2: int, mu_points: int, d_theta, piv: np.ndarray,
                  KmeansMaxIter_ISDF: int, layout: int = THETA_ROWS,
                  options: Options | None = None) -> Report:
    """The reference's p-rank GPU ISDF() for this rank (isdf_solve_sharded):
    d_psirow holds the rank's grid rows (row_block), d_theta receives its
    theta rows (THETA_ROWS: count x mu) or the reference's column-cyclic block
    (THETA_CYCLIC: Ng x (mu / p + (rank < mu % p)))."""
    piv = _host_int32(piv, domain.NumGridTotal())
    d = domain._c()
    o = (options or Options())._c()
    r = _Report()
    _check(lib().isdf_solve_sharded(comm._h, ctypes.byref(d), _dptr(d_psirow), nocc, nstate, nv1,
                                    nc1, nv2, nc2, mu_points, _dptr(d_theta), layout,
                                    piv.ctypes.data, KmeansMaxIter_ISDF, ctypes.byref(o),
                                    ctypes.byref(r)))
    return _report(r)


def kmeans_select_sharded(comm: Comm, domain: Domain, d_w, mu: int, max_iter: int,
                          rand_seed: int = -1):
    """This rank's part of the p-rank K-means selection from the full weight
    vector; returns (piv int32[Ng], rk_eff, iterations, npt), the same on every rank."""
    n = domain.NumGridTotal()
    piv = np.zeros(n, dtype=np.int32)
    out = (ctypes.c_int * 3)()
    d = domain._c()
    _check(lib().isdf_kmeans_select_sharded(comm._h, ctypes.byref(d), _dptr(d_w), mu, max_iter,
                                            rand_seed, piv.ctypes.data, ctypes.addressof(out),
                                            ctypes.addressof(out) + 4, ctypes.addressof(out) + 8))
    return piv, out[0], out[1], out[2]
