"""Continuous-batching server: a mix of systems of different grid sizes and
mu, submitted while others run, gives for every request exactly what a solve
of that request alone gives (bit-identical theta and piv, FP64 and mixed,
with the small requests' selections batched into shared launches and with
batching off); solves overlap (peak concurrency > 1); admission by device
footprint lets a large request wait while small ones pass, without starving
it; a queued request can be cancelled."""
import numpy as np
import pytest

from conftest import load_golden

import libisdf_b200 as isdf
from libisdf_b200 import synth

pytestmark = pytest.mark.gpu


def _requests(torch):
    reqs = []
    for name in ["small_s1s2", "small_mu0", "si8_example", "small_iters0"]:
        g = load_golden(name)
        reqs.append(dict(psi=g["psi"], ng=tuple(int(x) for x in g["ng"]),
                         length=tuple(float(x) for x in g["length"]),
                         a=(int(g["nocc"]), int(g["nv1"]), int(g["nc1"]), int(g["nv2"]),
                            int(g["nc2"])), mu=int(g["rk_requested"]), iters=int(g["iters"])))
    s = synth.SI8
    for seed in (100, 101):
        reqs.append(dict(psi=synth.shape_orbitals(s, seed), ng=(s.n,) * 3, length=(s.length,) * 3,
                         a=(s.nocc, s.nv1, s.nc1, s.nv2, s.nc2), mu=s.mu, iters=s.kmeans_iters))
    for r in reqs:
        r["d_psi"] = torch.from_numpy(np.ascontiguousarray(r["psi"].T)).cuda()
    return reqs


def _alone(torch, r, prec):
    d_theta = torch.zeros((r["mu"], r["psi"].shape[0]), dtype=torch.float64, device="cuda")
    piv = np.zeros(r["psi"].shape[0], dtype=np.int32)
    isdf.ISDF(r["d_psi"], isdf.Domain(length=r["length"], num_grid=r["ng"]), r["a"][0],
              r["psi"].shape[1], *r["a"][1:], r["mu"], d_theta, piv, r["iters"],
              options=isdf.Options(precision=prec, rand_seed=1))
    torch.cuda.synchronize()
    return d_theta.cpu().numpy(), piv


@pytest.mark.parametrize("prec,batch", [(isdf.PRECISION_FP64, 32), (isdf.PRECISION_MIXED, 32),
                                        (isdf.PRECISION_FP64, 0)])
def test_mix_equals_alone(torch_cuda, prec, batch):
    torch = torch_cuda
    reqs = _requests(torch)
    alone = [_alone(torch, r, prec) for r in reqs]
    with isdf.Server(slots=3, batch_small=batch) as srv:
        outs = []
        for rep in range(2):  # every request twice, interleaved
            for r in reqs:
                d_theta = torch.full((r["mu"], r["psi"].shape[0]), float("nan"),
                                     dtype=torch.float64, device="cuda")
                piv = np.zeros(r["psi"].shape[0], dtype=np.int32)
                t = srv.submit(r["d_psi"], isdf.Domain(length=r["length"], num_grid=r["ng"]),
                               r["a"][0], r["psi"].shape[1], *r["a"][1:], r["mu"], d_theta, piv,
                               r["iters"], options=isdf.Options(precision=prec, rand_seed=1))
                outs.append((t, d_theta, piv, len(outs) % len(reqs)))
        for t, d_theta, piv, k in outs:
            status, rep = srv.wait(t, 120000.0)
            assert status == isdf.ISDF_OK
            th_alone, piv_alone = alone[k]
            assert np.array_equal(piv, piv_alone)
            assert np.array_equal(d_theta.cpu().numpy(), th_alone)
        st = srv.stats()
    assert st["completed"] == 2 * len(reqs) and st["failed"] == 0
    assert st["peak_concurrency"] >= 2
    assert 0 < st["p50_ms"] <= st["p99_ms"]


def test_admission_budget_and_cancel(torch_cuda):
    torch = torch_cuda
    reqs = _requests(torch)
    big = reqs[-1]
    fp_big = isdf.workspace_bytes(big["psi"].shape[0], big["psi"].shape[1], big["mu"])
    # room for the large request alone, not for it plus another large one
    with isdf.Server(slots=4, hbm_budget_bytes=int(fp_big * 1.6), max_skips=4) as srv:
        tickets = []
        for r in reqs[::-1] + reqs:
            d_theta = torch.zeros((r["mu"], r["psi"].shape[0]), dtype=torch.float64,
                                  device="cuda")
            piv = np.zeros(r["psi"].shape[0], dtype=np.int32)
            tickets.append(srv.submit(r["d_psi"], isdf.Domain(length=r["length"],
                                                              num_grid=r["ng"]),
                                      r["a"][0], r["psi"].shape[1], *r["a"][1:], r["mu"],
                                      d_theta, piv, r["iters"]))
        last = srv.submit(reqs[0]["d_psi"], isdf.Domain(length=reqs[0]["length"],
                                                        num_grid=reqs[0]["ng"]),
                          reqs[0]["a"][0], reqs[0]["psi"].shape[1], *reqs[0]["a"][1:],
                          reqs[0]["mu"], torch.zeros((reqs[0]["mu"], reqs[0]["psi"].shape[0]),
                                                     dtype=torch.float64, device="cuda"),
                          np.zeros(reqs[0]["psi"].shape[0], dtype=np.int32), reqs[0]["iters"])
        cancelled = True
        try:
            srv.cancel(last)
        except isdf.IsdfError:
            cancelled = False  # it had already started
        for t in tickets:
            status, _ = srv.wait(t, 120000.0)
            assert status == isdf.ISDF_OK
        status, _ = srv.wait(last, 120000.0)
        assert status == (isdf.ISDF_ERR_CANCELLED if cancelled else isdf.ISDF_OK)
        st = srv.stats()
    assert st["peak_bytes"] <= int(fp_big * 1.6)
    assert st["completed"] >= len(tickets)
