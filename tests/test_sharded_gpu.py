"""Grid-row sharded solve on the GPU. The ranks run as host threads of one
process on one GPU, joined by the in-process transport (isdf_comm_create_local):
their collectives are device copies ordered by stream events, and no kernel
waits on another rank, so p ranks on one GPU are safe. Checked:
  * the p-rank K-means selection against the reference's own KMEAN run as p
    MPI ranks (the fixture tests/golden/sharded_kmeans.npz, made by
    tests/golden/make_sharded_golden.py), the rank-sensitive grids included,
    and against the p-rank port at the Si8-like size;
  * the sharded solve's theta against the one-rank solve: its rows (bit for
    bit when the pivots agree, FP64 and mixed), the reference's column-cyclic
    layout, and the NCCL transport at one rank;
  * a rank that never reaches a collective: the others fail with
    ISDF_ERR_COMM after the group's timeout, on the host;
  * a rank whose own checks fail, or that was called with other arguments
    than rank 0: every rank fails at the agreement before the first exchange,
    without waiting for the timeout;
  * the callback transport (isdf_comm_create_callbacks, the path for a caller
    with its own collectives) with Python collectives over host threads: the
    same theta columns as the one-rank solve."""
import threading
import time

import numpy as np
import pytest

from conftest import load_golden, record_parity
from oracle import fit as ofit
from oracle import port

import libisdf_b200 as isdf
from libisdf_b200 import synth

pytestmark = pytest.mark.gpu


def run_ranks(size, fn, timeout_s=60.0):
    """fn(rank, comm) on `size` threads with an in-process group; returns the
    per-rank results (re-raises the first exception)."""
    comms = isdf.Comm.local_group(size, timeout_s=timeout_s)
    out, err = [None] * size, [None] * size

    def body(r):
        try:
            out[r] = fn(r, comms[r])
        except BaseException as e:  # noqa: BLE001 - handed to the main thread
            err[r] = e

    th = [threading.Thread(target=body, args=(r,)) for r in range(size)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for c in comms:
        c.close()
    for e in err:
        if e is not None:
            raise e
    return out


def test_kmeans_sharded_matches_p_rank_reference(torch_cuda):
    torch = torch_cuda
    g = load_golden("sharded_kmeans")
    names = [str(x) for x in g["names"]]
    sensitive = 0
    for name in names:
        w, ng, ln = g[f"{name}/w"], g[f"{name}/ng"], g[f"{name}/length"]
        mu, it = int(g[f"{name}/mu"]), int(g[f"{name}/iters"])
        dom = isdf.Domain(length=tuple(ln), num_grid=tuple(int(x) for x in ng))
        d_w = torch.from_numpy(np.ascontiguousarray(w)).cuda()
        for p in (1, 2, 3, 4):
            res = run_ranks(p, lambda r, c: isdf.kmeans_select_sharded(c, dom, d_w, mu, it,
                                                                       rand_seed=1))
            for piv, rk, its, _ in res:
                assert np.array_equal(piv, g[f"{name}/piv{p}"]), (name, p)
                assert (rk, its) == (int(g[f"{name}/rk{p}"]), int(g[f"{name}/it{p}"])), (name, p)
        sensitive += any(not np.array_equal(g[f"{name}/piv{p}"], g[f"{name}/piv1"])
                         for p in (2, 3, 4))
    record_parity("sharded K-means", "fixture cases bit-exact at p = 1..4 (rank-sensitive)",
                  f"{len(names)} ({sensitive})")


@pytest.mark.parametrize("p", [2, 3])
def test_kmeans_sharded_si8(torch_cuda, p):
    """Si8-like shape (40^3 grid, mu = 320, 100 iterations): the p-rank
    selection against the p-rank port, bit for bit."""
    torch = torch_cuda
    s = synth.SI8
    psi = synth.shape_orbitals(s, 0)
    w = port.weight(psi, s.nocc, s.nv1, s.nc1, s.nv2, s.nc2)
    dom = isdf.Domain(length=(s.length,) * 3, num_grid=(s.n,) * 3)
    d_w = torch.from_numpy(w).cuda()
    res = run_ranks(p, lambda r, c: isdf.kmeans_select_sharded(c, dom, d_w, s.mu, s.kmeans_iters))
    want = port.kmeans_ranks(w, (s.n,) * 3, (s.length,) * 3, s.mu, s.kmeans_iters, p)
    for piv, rk, its, _ in res:
        assert np.array_equal(piv, want[0])
        assert (rk, its) == want[1:]


def _split_rows(torch, psi, p, r):
    start, cnt = isdf.row_block(psi.shape[0], p, r)
    return start, cnt, torch.from_numpy(np.ascontiguousarray(psi[start:start + cnt].T)).cuda()


def _single(torch, psi, dom, a, mu, iters, opts):
    d_psi = torch.from_numpy(np.ascontiguousarray(psi.T)).cuda()
    d_th = torch.empty((mu, psi.shape[0]), dtype=torch.float64, device="cuda")
    piv = np.zeros(psi.shape[0], dtype=np.int32)
    rep = isdf.ISDF(d_psi, dom, a[0], psi.shape[1], *a[1:], mu, d_th, piv, iters, options=opts)
    return np.asfortranarray(d_th.cpu().numpy().T), piv, rep


@pytest.mark.parametrize("precision", [isdf.PRECISION_FP64, isdf.PRECISION_MIXED])
@pytest.mark.parametrize("case", ["small_s1s2", "si8"])
def test_solve_sharded_rows(torch_cuda, precision, case):
    """theta rows of the p-rank solve (THETA_ROWS) against the one-rank solve:
    equal pivots, and bit-identical rows (every element is the same products
    in the same order), FP64 and mixed; the S1 != S2 window included."""
    torch = torch_cuda
    if case == "si8":
        s = synth.SI8
        psi = synth.shape_orbitals(s, 0)
        a = (s.nocc, s.nv1, s.nc1, s.nv2, s.nc2)
        ng, ln, mu, iters = (s.n,) * 3, (s.length,) * 3, s.mu, s.kmeans_iters
    else:
        g = load_golden(case)
        psi = g["psi"]
        a = (int(g["nocc"]), int(g["nv1"]), int(g["nc1"]), int(g["nv2"]), int(g["nc2"]))
        ng, ln = tuple(int(x) for x in g["ng"]), tuple(g["length"])
        mu, iters = int(g["rk_requested"]), int(g["iters"])
    dom = isdf.Domain(length=ln, num_grid=ng)
    opts = isdf.Options(precision=precision)
    th1, piv1, rep1 = _single(torch, psi, dom, a, mu, iters, opts)
    for p in (2, 3):
        def rank(r, c):
            start, cnt, d_rows = _split_rows(torch, psi, p, r)
            d_th = torch.full((mu, cnt), float("nan"), dtype=torch.float64, device="cuda")
            piv = np.zeros(psi.shape[0], dtype=np.int32)
            rep = isdf.solve_sharded(c, d_rows, dom, a[0], psi.shape[1], *a[1:], mu, d_th, piv,
                                     iters, layout=isdf.THETA_ROWS, options=opts)
            return start, cnt, d_th.cpu().numpy().T, piv, rep
        res = run_ranks(p, rank)
        for start, cnt, rows, piv, rep in res:
            assert np.array_equal(piv, piv1), (case, p)
            assert rep.rk_eff == rep1.rk_eff and rep.kmeans_iters == rep1.kmeans_iters
            assert np.array_equal(rows, th1[start:start + cnt]), (case, p, start)
    record_parity(f"sharded solve {case} {'mixed' if precision else 'FP64'}",
                  "theta rows vs one rank (p = 2, 3)", "bit-identical")


def test_solve_sharded_cyclic_layout_and_oracle(torch_cuda):
    """The reference's column-cyclic d_thetaCol (GPU_AlltoallBackward,
    src/common/utility.cpp:444-526): rank r holds columns r, r + p, ... of
    theta over all Ng rows, mu not a multiple of p; theta against the oracle's
    FP64 fit on the reference's own case."""
    torch = torch_cuda
    g = load_golden("small_mu0")
    psi = g["psi"]
    a = (int(g["nocc"]), int(g["nv1"]), int(g["nc1"]), int(g["nv2"]), int(g["nc2"]))
    ng, ln = tuple(int(x) for x in g["ng"]), tuple(g["length"])
    mu, iters = 46, int(g["iters"])
    dom = isdf.Domain(length=ln, num_grid=ng)
    th1, piv1, rep1 = _single(torch, psi, dom, a, mu, iters, isdf.Options())
    for p in (2, 3, 4):
        def rank(r, c):
            start, cnt, d_rows = _split_rows(torch, psi, p, r)
            w = mu // p + (1 if r < mu % p else 0)
            d_th = torch.full((w, psi.shape[0]), float("nan"), dtype=torch.float64, device="cuda")
            piv = np.zeros(psi.shape[0], dtype=np.int32)
            isdf.solve_sharded(c, d_rows, dom, a[0], psi.shape[1], *a[1:], mu, d_th, piv, iters,
                               layout=isdf.THETA_CYCLIC)
            return d_th.cpu().numpy().T, piv
        res = run_ranks(p, rank)
        for r, (cols, piv) in enumerate(res):
            assert np.array_equal(piv, piv1)
            assert np.array_equal(cols, th1[:, r::p]), (p, r)
    th_o = ofit.getbasis(psi, *a, rep1.rk_eff, piv1)
    fd = ofit.fitted_densities(th1[:, :rep1.rk_eff], psi, *a, rep1.rk_eff, piv1)
    fd_o = ofit.fitted_densities(th_o, psi, *a, rep1.rk_eff, piv1)
    err = ofit.rel(fd, fd_o)
    record_parity("sharded solve small_mu0", "fitted densities vs oracle", err, 1e-10)
    assert err <= 1e-10


def test_nccl_transport_one_rank(torch_cuda):
    """The NCCL transport at world size 1 (the only size one GPU allows) runs
    the sharded path end to end and equals the one-rank solve bit for bit."""
    torch = torch_cuda
    g = load_golden("small_s1s2")
    psi = g["psi"]
    a = (int(g["nocc"]), int(g["nv1"]), int(g["nc1"]), int(g["nv2"]), int(g["nc2"]))
    dom = isdf.Domain(length=tuple(g["length"]), num_grid=tuple(int(x) for x in g["ng"]))
    mu, iters = int(g["rk_requested"]), int(g["iters"])
    th1, piv1, _ = _single(torch, psi, dom, a, mu, iters, isdf.Options())
    comm = isdf.Comm.nccl(isdf.nccl_unique_id(), 0, 1)
    try:
        for layout in (isdf.THETA_ROWS, isdf.THETA_CYCLIC):
            d_th = torch.full((mu, psi.shape[0]), float("nan"), dtype=torch.float64, device="cuda")
            piv = np.zeros(psi.shape[0], dtype=np.int32)
            isdf.solve_sharded(comm, torch.from_numpy(np.ascontiguousarray(psi.T)).cuda(), dom,
                               a[0], psi.shape[1], *a[1:], mu, d_th, piv, iters, layout=layout)
            assert np.array_equal(piv, piv1)
            assert np.array_equal(d_th.cpu().numpy().T, th1)
    finally:
        comm.close()


def test_missing_rank_fails_on_the_host(torch_cuda):
    """A rank that never reaches the first collective: the other ranks'
    solves return ISDF_ERR_COMM once the group's 1 s timeout runs out; no
    kernel waits on a rank, so the GPU is untouched by the failure."""
    torch = torch_cuda
    g = load_golden("small_s1s2")
    psi = g["psi"]
    a = (int(g["nocc"]), int(g["nv1"]), int(g["nc1"]), int(g["nv2"]), int(g["nc2"]))
    dom = isdf.Domain(length=tuple(g["length"]), num_grid=tuple(int(x) for x in g["ng"]))
    mu, iters, p = int(g["rk_requested"]), int(g["iters"]), 3

    def rank(r, c):
        if r == 2:
            return None  # this rank leaves before its first collective
        start, cnt, d_rows = _split_rows(torch, psi, p, r)
        d_th = torch.empty((mu, cnt), dtype=torch.float64, device="cuda")
        piv = np.zeros(psi.shape[0], dtype=np.int32)
        with pytest.raises(isdf.IsdfError) as ei:
            isdf.solve_sharded(c, d_rows, dom, a[0], psi.shape[1], *a[1:], mu, d_th, piv, iters)
        return ei.value.code

    codes = run_ranks(p, rank, timeout_s=1.0)
    assert codes[:2] == [isdf.ISDF_ERR_COMM] * 2
    torch.cuda.synchronize()  # the context is intact
    th1, piv1, _ = _single(torch, psi, dom, a, mu, iters, isdf.Options())
    assert np.isfinite(th1).all()


def _small_case():
    g = load_golden("small_s1s2")
    psi = g["psi"]
    a = (int(g["nocc"]), int(g["nv1"]), int(g["nc1"]), int(g["nv2"]), int(g["nc2"]))
    dom = isdf.Domain(length=tuple(g["length"]), num_grid=tuple(int(x) for x in g["ng"]))
    return psi, a, dom, int(g["rk_requested"]), int(g["iters"])


def _solve_code(torch, c, psi, a, dom, p, r, mu, iters, layout=isdf.THETA_ROWS):
    start, cnt, d_rows = _split_rows(torch, psi, p, r)
    shape = (mu, cnt) if layout == isdf.THETA_ROWS else (mu // p + 1, psi.shape[0])
    d_th = torch.empty(shape, dtype=torch.float64, device="cuda")
    piv = np.zeros(psi.shape[0], dtype=np.int32)
    with pytest.raises(isdf.IsdfError) as ei:
        isdf.solve_sharded(c, d_rows, dom, a[0], psi.shape[1], *a[1:], mu, d_th, piv, iters,
                           layout=layout)
    return ei.value.code, str(ei.value)


@pytest.mark.parametrize("layout", [isdf.THETA_ROWS, isdf.THETA_CYCLIC])
def test_failed_rank_fails_every_rank(torch_cuda, layout):
    """Rank 1 is called with a negative K-means iteration cap: it returns
    ISDF_ERR_ARG, and ranks 0 and 2 return ISDF_ERR_COMM naming rank 1, at the
    agreement before the first exchange, well inside the group's 30 s timeout."""
    torch = torch_cuda
    psi, a, dom, mu, iters = _small_case()
    p = 3

    def rank(r, c):
        return _solve_code(torch, c, psi, a, dom, p, r, mu, -1 if r == 1 else iters, layout)

    t0 = time.monotonic()
    out = run_ranks(p, rank, timeout_s=30.0)
    took = time.monotonic() - t0
    assert [o[0] for o in out] == [isdf.ISDF_ERR_COMM, isdf.ISDF_ERR_ARG, isdf.ISDF_ERR_COMM]
    assert "negative K-means iteration cap" in out[1][1]
    assert all("rank 1 failed" in out[q][1] for q in (0, 2))
    assert took < 20.0, took
    th1, piv1, _ = _single(torch, psi, dom, a, mu, iters, isdf.Options())
    assert np.isfinite(th1).all()  # the context is intact


def test_ranks_with_other_arguments_fail(torch_cuda):
    """Rank 2 asks for one interpolation point fewer than ranks 0 and 1: every
    rank returns ISDF_ERR_ARG before the first exchange. The sharded K-means
    selection checks its arguments the same way."""
    torch = torch_cuda
    psi, a, dom, mu, iters = _small_case()
    p = 3

    def rank(r, c):
        return _solve_code(torch, c, psi, a, dom, p, r, mu - 1 if r == 2 else mu, iters)

    out = run_ranks(p, rank, timeout_s=30.0)
    assert [o[0] for o in out] == [isdf.ISDF_ERR_ARG] * 3
    assert all("other arguments than rank 0" in o[1] for o in out)

    w = torch.from_numpy(load_golden("small_s1s2")["weight"].copy()).cuda()

    def sel(r, c):
        with pytest.raises(isdf.IsdfError) as ei:
            isdf.kmeans_select_sharded(c, dom, w, mu, iters + (r == 0))
        return ei.value.code

    assert run_ranks(2, sel, timeout_s=30.0) == [isdf.ISDF_ERR_ARG] * 2


class _DeviceBytes:
    """`n` bytes of device memory at a raw address, for torch.as_tensor."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "|u1", "data": (ptr, False),
                                         "version": 2, "strides": None}


class _ThreadCollectives:
    """A caller's own collectives for ranks on host threads of one process: the
    sender's stream is synchronised before its buffer is published, every
    rank copies what it needs on its own stream and synchronises it, and a
    second barrier keeps send buffers alive until all ranks have read them."""

    def __init__(self, torch, size):
        self.torch, self.size = torch, size
        self.barrier = threading.Barrier(size, timeout=30.0)
        self.slots = [None] * size
        self.calls = [0] * size

    def _bytes(self, ptr, n):
        return self.torch.as_tensor(_DeviceBytes(ptr, n), device="cuda")

    def _run(self, rank, stream, slot, copies):
        torch = self.torch
        s = torch.cuda.ExternalStream(stream)
        s.synchronize()
        self.slots[rank] = slot
        self.barrier.wait()
        with torch.cuda.stream(s):
            for dst, src, n in copies():
                if n:
                    self._bytes(dst, n).copy_(self._bytes(src, n))
        s.synchronize()
        self.barrier.wait()
        self.calls[rank] += 1

    def comm(self, rank):
        def allgatherv(d_send, send_bytes, d_recv, counts, displs, stream):
            self._run(rank, stream, d_send,
                      lambda: [(d_recv + displs[q], self.slots[q], counts[q])
                               for q in range(self.size)])

        def alltoallv(d_send, scounts, sdispls, d_recv, rcounts, rdispls, stream):
            self._run(rank, stream, (d_send, sdispls),
                      lambda: [(d_recv + rdispls[q], self.slots[q][0] + self.slots[q][1][rank],
                                rcounts[q]) for q in range(self.size)])

        return isdf.Comm.callbacks(allgatherv, alltoallv, rank, self.size)


def test_callback_transport(torch_cuda):
    """Two ranks whose collectives are the caller's own (Python callbacks over
    host threads) give the one-rank solve's theta columns in the reference's
    cyclic layout, and its piv."""
    torch = torch_cuda
    g = load_golden("small_mu0")
    psi = g["psi"]
    a = (int(g["nocc"]), int(g["nv1"]), int(g["nc1"]), int(g["nv2"]), int(g["nc2"]))
    dom = isdf.Domain(length=tuple(g["length"]), num_grid=tuple(int(x) for x in g["ng"]))
    mu, iters, p = 46, int(g["iters"]), 2
    th1, piv1, _ = _single(torch, psi, dom, a, mu, iters, isdf.Options())
    coll = _ThreadCollectives(torch, p)
    comms = [coll.comm(r) for r in range(p)]
    out, err = [None] * p, [None] * p

    def body(r):
        try:
            start, cnt, d_rows = _split_rows(torch, psi, p, r)
            w = mu // p + (1 if r < mu % p else 0)
            d_th = torch.full((w, psi.shape[0]), float("nan"), dtype=torch.float64, device="cuda")
            piv = np.zeros(psi.shape[0], dtype=np.int32)
            isdf.solve_sharded(comms[r], d_rows, dom, a[0], psi.shape[1], *a[1:], mu, d_th, piv,
                               iters, layout=isdf.THETA_CYCLIC)
            out[r] = (d_th.cpu().numpy().T, piv)
        except BaseException as e:  # noqa: BLE001 - handed to the main thread
            err[r] = e
            coll.barrier.abort()

    th = [threading.Thread(target=body, args=(r,)) for r in range(p)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for c in comms:
        c.close()
    for e in err:
        if e is not None:
            raise e
    for r, (cols, piv) in enumerate(out):
        assert np.array_equal(piv, piv1)
        assert np.array_equal(cols, th1[:, r::p]), r
    assert coll.calls[0] == coll.calls[1] > 2
    record_parity("sharded solve small_mu0, callback transport",
                  "theta columns vs one rank (p = 2)", "bit-identical")
