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
    ISDF_ERR_COMM after the group's timeout, on the host."""
import threading

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
