"""Generates the golden fixtures in tests/golden/ by running the reference's own
CPU code (oracle/_ref/libisdf_ref.so, built by oracle/build_ref.sh from the
reference sources with single-rank shims).

    python tests/golden/make_golden.py [--reference-data DIR]

DIR defaults to the reference checkout's examples/si8/data (psirow0/psirow1,
the only data the reference ships). Each case stores its inputs (psi, grid,
state windows, mu, iteration cap) and the reference's outputs: the weight,
piv, the effective mu, the Lloyd iteration count, theta (small cases) or its
first columns, and the check's fit / Coulomb errors where computed.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from libisdf_b200 import synth  # noqa: E402
from oracle import ref  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def read_psirow(path):
    with open(path) as f:
        rows = int(f.readline())
        cols = int(f.readline())
        vals = np.array(f.read().split(), dtype=np.float64)
    return vals.reshape(cols, rows).T  # stored column by column


def save(name, psi, ng, length, nocc, nv1, nc1, nv2, nc2, mu, iters, theta_cols=None,
         check=False, store_psi=True, rand_seed=1, extra=None):
    psi = np.asfortranarray(psi)
    rk_req = mu if mu else ref.iround(np.sqrt((nc1 + nv1) * (nc2 + nv2)) * 8.0)
    piv, rk, it, w = ref.kmeans_piv(psi, ng, length, nocc, nv1, nc1, nv2, nc2, rk_req, iters,
                                    rand_seed=rand_seed, cross_check=True)
    out = dict(ng=np.array(ng, dtype=np.int32), length=np.array(length, dtype=np.float64),
               nocc=nocc, nv1=nv1, nc1=nc1, nv2=nv2, nc2=nc2, mu_points=mu, rk_requested=rk_req,
               iters=iters, rand_seed=rand_seed, piv=piv, rk_eff=rk, n_iter=it, weight=w,
               psi_sha256=synth.sha256(psi))
    if store_psi:
        out["psi"] = psi
    fit_ok = it >= 0  # the npt < mu early return leaves piv unsuitable for a fit
    if fit_ok:
        th = ref.getbasis(psi, ng, length, nocc, nv1, nc1, nv2, nc2, rk, piv)
        if theta_cols is None:
            out["theta"] = th
        else:
            out["theta_cols"] = np.ascontiguousarray(th[:, :theta_cols])
        if check:
            fe, ce = ref.checkcode(psi, ng, length, nocc, nv1, nc1, nv2, nc2, rk, piv, th)
            out["fit_err"] = fe
            out["coul_err"] = ce
    if extra:
        out.update(extra)
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **out)
    print(f"{name}: Ng={np.prod(ng)} rk={rk_req}->{rk} iters={it}"
          + (f" fit_err={out.get('fit_err')} coul_err={out.get('coul_err')}" if check else ""))


def localized_orbitals(n, length, nstate, seed, alpha):
    """Very narrow Gaussians: most grid points fall below the 1e-8 weight filter."""
    rng = np.random.default_rng(seed)
    h = length / n
    g = synth.grid_coords(n, length)
    centres = rng.uniform(0, length, size=(2, 3))
    psi = np.zeros((g.shape[0], nstate))
    for s in range(nstate):
        c = centres[s % 2]
        d = g - c
        psi[:, s] = np.exp(-alpha * (d * d).sum(1)) * (1.0 + 0.1 * s * d[:, 0] / h)
    q, _ = np.linalg.qr(psi)
    return np.asfortranarray(q)


def main():
    ap = argparse.ArgumentParser()
    root = os.environ.get("ISDF_REFERENCE_ROOT", "")
    ap.add_argument("--reference-data",
                    default=os.path.join(root, "examples", "si8", "data") if root else None,
                    required=not root,
                    help="the reference's examples/si8/data (default: under $ISDF_REFERENCE_ROOT)")
    a = ap.parse_args()
    if not ref.available():
        sys.exit("oracle/_ref/libisdf_ref.so is missing: run oracle/build_ref.sh first")

    # 1. The reference's own example: Si8, 16^3, 35 states, Nv=16, Nc=0, mu=192,
    #    500 iterations (examples/si8/readpsi.cpp:128-176,217-218), the two rank
    #    blocks stacked into one rank.
    p0 = read_psirow(os.path.join(a.reference_data, "psirow0"))
    p1 = read_psirow(os.path.join(a.reference_data, "psirow1"))
    psi = np.vstack([p0, p1])
    save("si8_example", psi, (16, 16, 16), (10.216, 10.216, 10.216), 16, 16, 0, 16, 0, 192, 500,
         theta_cols=8, check=True)

    # 2. S1 != S2 (the two-GEMM branch, isdf-gpu.cpp:231-259), small synthetic.
    psi = synth.orbitals(12, 1, 12, seed=11)
    save("small_s1s2", psi, (12, 12, 12), (synth.A_SI,) * 3, 6, 6, 6, 3, 2, 40, 50, check=True)

    # 3. Non-cubic grid and lengths, mu_points = 0 (default mu formula).
    rng = np.random.default_rng(12)
    raw = rng.standard_normal((10 * 12 * 14, 6)) * np.exp(
        -0.5 * rng.uniform(0, 3, size=(10 * 12 * 14, 1)))
    psi = np.asfortranarray(np.linalg.qr(raw)[0])
    save("small_mu0", psi, (10, 12, 14), (9.0, 10.0, 11.0), 3, 3, 3, 3, 3, 0, 30, check=True)

    # 4. KmeansMaxIter = 0: the initial assignment feeds the final argmin.
    psi = synth.orbitals(10, 1, 8, seed=13)
    save("small_iters0", psi, (10, 10, 10), (synth.A_SI,) * 3, 4, 4, 4, 4, 4, 30, 0)

    # 5. npt < mu: the early-return branch with the shuffled tail.
    psi = localized_orbitals(10, 10.0, 4, seed=14, alpha=40.0)
    save("small_early", psi, (10, 10, 10), (10.0,) * 3, 2, 2, 2, 2, 2, 200, 10)

    # 6. Si8-like synthetic (BASELINE config 0 shape): outputs only, psi is
    #    regenerated from its seed (the stored SHA-256 says whether the bits
    #    match on the machine that regenerates it).
    s = synth.SI8
    psi = synth.shape_orbitals(s, 0)
    save("si8_synth_seed0", psi, (s.n,) * 3, (s.length,) * 3, s.nocc, s.nv1, s.nc1, s.nv2, s.nc2,
         s.mu, s.kmeans_iters, theta_cols=4, store_psi=False)


if __name__ == "__main__":
    main()
