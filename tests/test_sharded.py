"""Grid-row sharding on the CPU: the reference's block rule, the p-rank
oracle against the reference's own KMEAN run as p ranks, the p-rank
restatement run as real gloo ranks (world size 2 and 3), and the NCCL
unique-id hand-over through torch.distributed. No GPU."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import load_golden

import libisdf_b200 as isdf
from oracle import port, ref

RANKS = (1, 2, 3, 4)


def _cases():
    g = load_golden("sharded_kmeans")
    return g, [str(x) for x in g["names"]]


def test_row_block_is_the_reference_rule():
    """isdf_row_block against the ntotLocal / displacement rule of
    src/common/isdf.cpp:137-141 and src/cuda/isdf-gpu.cpp:64-78."""
    for n in (1, 7, 8, 1000, 1259712, 64001):
        for p in range(1, 9):
            if p > n:
                continue
            blk = n // p
            pos = 0
            for r in range(p):
                local = blk + (1 if r < n % p else 0)
                disp = r * (blk + 1) if r < n % p else (n % p) * (blk + 1) + (r - n % p) * blk
                assert isdf.row_block(n, p, r) == (disp, local)
                assert disp == pos
                pos += local
            assert pos == n
    with pytest.raises(isdf.IsdfError):
        isdf.row_block(10, 2, 2)


def test_port_ranks_matches_fixture():
    """oracle/kmeans_port.cpp's p-rank restatement reproduces the reference's
    p-rank piv, mu and iteration count on every fixture case, including the
    rank-sensitive grids where p ranks select other points than one rank."""
    g, names = _cases()
    sensitive = 0
    for name in names:
        w, ng, ln = g[f"{name}/w"], g[f"{name}/ng"], g[f"{name}/length"]
        mu, it = int(g[f"{name}/mu"]), int(g[f"{name}/iters"])
        for p in RANKS:
            piv, rk, its = port.kmeans_ranks(w, ng, ln, mu, it, p)
            assert np.array_equal(piv, g[f"{name}/piv{p}"]), (name, p)
            assert (rk, its) == (int(g[f"{name}/rk{p}"]), int(g[f"{name}/it{p}"]))
        sensitive += any(not np.array_equal(g[f"{name}/piv{p}"], g[f"{name}/piv1"])
                         for p in RANKS[1:])
    assert sensitive >= 8


@pytest.mark.skipif(not ref.available_ranks(), reason="oracle/_ref not built")
def test_p_rank_reference_live():
    """The reference's own KMEAN as p forked ranks (oracle/_ref) gives the
    fixture again, and one rank of it equals the one-rank golden piv."""
    g, names = _cases()
    for name in names[:3] + ["small_s1s2"]:
        w, ng, ln = g[f"{name}/w"], g[f"{name}/ng"], g[f"{name}/length"]
        mu, it = int(g[f"{name}/mu"]), int(g[f"{name}/iters"])
        for p in RANKS:
            piv, rk, its = ref.kmeans_ranks(w, ng, ln, mu, it, p)
            assert np.array_equal(piv, g[f"{name}/piv{p}"]), (name, p)
    one = load_golden("small_s1s2")
    assert np.array_equal(g["small_s1s2/piv1"], one["piv"])


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port_ = s.getsockname()[1]
    s.close()
    return port_


def _gloo_rank(rank, size, port_, names, q):
    import torch.distributed as dist

    from oracle import kmeans_sharded

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port_)
    dist.init_process_group("gloo", rank=rank, world_size=size,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        g = load_golden("sharded_kmeans")
        out = {}
        for name in names:
            w, ng, ln = g[f"{name}/w"], g[f"{name}/ng"], g[f"{name}/length"]
            mu, it = int(g[f"{name}/mu"]), int(g[f"{name}/iters"])
            piv, rk, its = kmeans_sharded.kmeans_rank(w, ng, ln, mu, it)
            out[name] = (np.array_equal(piv, g[f"{name}/piv{size}"]),
                         (rk, its) == (int(g[f"{name}/rk{size}"]), int(g[f"{name}/it{size}"])))
        # the NCCL id made on rank 0 reaches every rank intact
        nid = isdf.share_nccl_unique_id()
        ids = [None] * size
        dist.all_gather_object(ids, nid)
        out["nccl_id"] = (len(nid) == 128 and all(x == ids[0] for x in ids), True)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("size", [2, 3])
def test_p_rank_restatement_over_gloo(size):
    """The p-rank KMEAN restated with real collectives: `size` gloo processes
    exchange partial sums by all-gather and combine them in binomial order;
    every rank's piv equals the reference's p-rank piv."""
    g, names = _cases()
    names = [n for n in names if n != "small_early"]  # its npt < mu branch draws from rand()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port_ = _free_port()
    procs = [ctx.Process(target=_gloo_rank, args=(r, size, port_, names, q)) for r in range(size)]
    for pr in procs:
        pr.start()
    results = {}
    try:
        for _ in range(size):
            r, out = q.get(timeout=240)
            results[r] = out
    finally:
        for pr in procs:
            pr.join(timeout=60)
            if pr.is_alive():
                pr.kill()
    assert sorted(results) == list(range(size))
    for r, out in results.items():
        for name, (same_piv, same_counts) in out.items():
            assert same_piv and same_counts, (r, name)
