"""Generates tests/golden/sharded_kmeans.npz: the reference's own KMEAN
(src/common/utility.cpp:631-988) run as p = 1, 2, 3, 4 MPI ranks
(oracle/_ref/libisdf_ref_mp.so: forked ranks over the shared-memory MPI
stand-in of oracle/shims_mp, reductions in binomial-tree order).

    python tests/golden/make_sharded_golden.py

Cases:
  * rank-sensitive grids: weights w(x, y, z) = f(x) g(y) h(z) with each factor
    mirror-symmetric, mu = 1 or 2, so that a centroid sits on the bisector
    of two grid points up to rounding; the order in which the ranks' partial
    sums are combined then decides which point is nearest, and the p-rank piv
    differs from the one-rank piv. Drawn from a seeded generator and kept
    only when some p gives a piv different from p = 1;
  * the reference's own small cases (tests/golden/small_*.npz, the Si8
    example) at every p.
For every case and p the file holds piv, the effective mu and the Lloyd
iteration count, and the script checks that oracle/kmeans_port.cpp's p-rank
restatement gives the same.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import port, ref  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
RANKS = (1, 2, 3, 4)
ITERS = 10


def symmetric_cases(count, seed=11):
    rng = np.random.default_rng(seed)
    cases = []
    while len(cases) < count:
        dims = rng.integers(2, 7, 3)
        f = []
        for d in dims:
            h = rng.random((d + 1) // 2) + 0.1
            f.append(np.concatenate([h, h[::-1][d % 2:]])[:d])
        w = np.einsum("i,j,k->kji", f[0], f[1], f[2]).reshape(-1).copy()  # x fastest
        ng = np.array(dims, dtype=np.int32)
        ln = rng.uniform(3, 12, 3)
        mu = int(rng.integers(1, 3))
        p1 = port.kmeans_ranks(w, ng, ln, mu, ITERS, 1)
        if any(not np.array_equal(port.kmeans_ranks(w, ng, ln, mu, ITERS, p)[0], p1[0])
               for p in RANKS[1:] if p <= w.size):
            cases.append((f"sym{len(cases)}", w, ng, ln, mu, ITERS))
    return cases


def golden_cases():
    out = []
    for name in ("small_s1s2", "small_mu0", "small_iters0", "small_early", "si8_example"):
        with np.load(os.path.join(OUT, name + ".npz")) as g:
            out.append((name, g["weight"].copy(), g["ng"].astype(np.int32), g["length"].copy(),
                        int(g["rk_requested"]), int(g["iters"])))
    return out


def main():
    if not ref.available_ranks():
        raise SystemExit("oracle/_ref/libisdf_ref_mp.so is missing: run oracle/build_ref.sh")
    data = {}
    names = []
    for name, w, ng, ln, mu, iters in symmetric_cases(8) + golden_cases():
        names.append(name)
        data[f"{name}/w"] = w
        data[f"{name}/ng"] = ng
        data[f"{name}/length"] = ln
        data[f"{name}/mu"] = np.int32(mu)
        data[f"{name}/iters"] = np.int32(iters)
        for p in RANKS:
            piv, rk, it = ref.kmeans_ranks(w, ng, ln, mu, iters, p)
            ppiv, prk, pit = port.kmeans_ranks(w, ng, ln, mu, iters, p)
            assert np.array_equal(piv, ppiv) and (rk, it) == (prk, pit), (name, p)
            data[f"{name}/piv{p}"] = piv
            data[f"{name}/rk{p}"] = np.int32(rk)
            data[f"{name}/it{p}"] = np.int32(it)
        diff = [p for p in RANKS[1:] if not np.array_equal(data[f"{name}/piv{p}"],
                                                           data[f"{name}/piv1"])]
        print(f"{name}: n={w.size} mu={mu} rk={data[f'{name}/rk1']} "
              f"iters={data[f'{name}/it1']} ranks giving another piv than p=1: {diff}")
    data["names"] = np.array(names)
    np.savez_compressed(os.path.join(OUT, "sharded_kmeans.npz"), **data)


if __name__ == "__main__":
    main()
