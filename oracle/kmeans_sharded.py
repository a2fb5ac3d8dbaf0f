"""Test infrastructure only (oracle): the reference's KMEAN as one rank of p,
in numpy, with the collectives over torch.distributed (gloo on CPU).

It restates src/common/utility.cpp:631-988 at world size p the way the
reference runs it: rank r owns the points [r n/p + min(r, n%p), + n/p +
(r < n%p)) of the n-long index list (zero tail included, :682-713), assigns
them ((dx*dx + dy*dy) + dz*dz, first minimum, :598-615, :579-595), folds its
centroid sums in its point order (:813-822); the ranks' partial sums meet in
an all-gather and are combined in binomial-tree order (the order of MPICH's
binomial MPI_Reduce, :825-826); the compaction of empty clusters and the
loop test follow :831-917; the nearest point of each centroid is each rank's
first minimum, then the smallest distance over the ranks with ties to the
smaller grid index (MPI_MINLOC, :926-969). Small cases only (it holds a
points x centroids distance block). Only tests import this module.
"""
from __future__ import annotations

import numpy as np


def _coords(t, ng, dx):
    nx, ny = int(ng[0]), int(ng[1])
    gx = (t % nx).astype(np.float64) * dx[0]
    gy = ((t % (nx * ny)).astype(np.float64) - gx / dx[0]) / nx * dx[1]
    gz = (t.astype(np.float64) - gx / dx[0] - gy / dx[1] * nx) / (nx * ny) * dx[2]
    return gx, gy, gz


def _dist(px, py, pz, cx, cy, cz):
    d1 = px[:, None] - cx[None, :]
    d2 = py[:, None] - cy[None, :]
    d3 = pz[:, None] - cz[None, :]
    return (d1 * d1 + d2 * d2) + d3 * d3


def _binomial(parts):
    """Combine the ranks' arrays: at step s = 1, 2, 4, ..., rank q takes in q + s."""
    parts = [p.copy() for p in parts]
    s = 1
    while s < len(parts):
        for q in range(0, len(parts) - s, 2 * s):
            parts[q] = parts[q] + parts[q + s]
        s *= 2
    return parts[0]


def kmeans_rank(w, ng, length, mu, max_iter, group=None):
    """This rank's part of the p-rank selection; every rank returns the same
    (piv int32[n], rk_eff, iterations). Cold start, mu <= kept points."""
    import torch
    import torch.distributed as dist

    rank, p = dist.get_rank(group), dist.get_world_size(group)
    w = np.asarray(w, dtype=np.float64)
    n = w.size
    maxw = max(0.0, float(w.max()))
    kept = np.nonzero(w > 1e-8 * maxw)[0]
    npt = kept.size
    if npt < mu:
        raise NotImplementedError("the npt < mu branch draws from rand(); not restated here")
    index = np.zeros(n, dtype=np.int64)
    index[:npt] = kept
    dx = [float(length[i]) / int(ng[i]) for i in range(3)]
    lo = rank * (n // p) + min(rank, n % p)
    cnt = n // p + (1 if rank < n % p else 0)
    idx = index[lo:lo + cnt]
    px, py, pz = _coords(idx, ng, dx)
    wl = w[idx]
    cx, cy, cz = (c.copy() for c in _coords(index[:mu], ng, dx))
    rk = mu

    def all_gather(arr):
        t = torch.from_numpy(np.ascontiguousarray(arr))
        out = [torch.empty_like(t) for _ in range(p)]
        dist.all_gather(out, t, group=group)
        return [o.numpy() for o in out]

    lab = np.argmin(_dist(px, py, pz, cx, cy, cz), axis=1)
    flag, s = n, 0
    while flag > 1e-5 * n and s < max_iter:
        part = np.zeros((4, rk))
        np.add.at(part[0], lab, wl)  # unbuffered: index order, one addition per point
        np.add.at(part[1], lab, wl * px)
        np.add.at(part[2], lab, wl * py)
        np.add.at(part[3], lab, wl * pz)
        tot = _binomial(all_gather(part))
        cntc, sx, sy, sz = (list(r) for r in tot)
        i = 0
        while i < rk:
            if cntc[i] != 0.0:
                sx[i], sy[i], sz[i] = sx[i] / cntc[i], sy[i] / cntc[i], sz[i] / cntc[i]
                i += 1
            else:
                rk -= 1
                sx[i], sy[i], sz[i], cntc[i] = sx[rk], sy[rk], sz[rk], cntc[rk]
        cx, cy, cz = (np.array(v[:rk]) for v in (sx, sy, sz))
        last = lab
        lab = np.argmin(_dist(px, py, pz, cx, cy, cz), axis=1)
        changed = np.array([int((last != lab).sum())], dtype=np.int64)
        flag = int(sum(int(c[0]) for c in all_gather(changed)))
        s += 1
    D = _dist(px, py, pz, cx, cy, cz)
    bi = np.argmin(D, axis=0)
    mine = np.stack([D[bi, np.arange(rk)], idx[bi].astype(np.float64)])
    best = None
    for q in all_gather(mine):
        if best is None:
            best = q.copy()
            continue
        take = (q[0] < best[0]) | ((q[0] == best[0]) & (q[1] < best[1]))
        best[:, take] = q[:, take]
    sel = np.unique(best[1].astype(np.int64))
    rk = sel.size
    piv = np.empty(n, dtype=np.int32)
    piv[:rk] = sel
    rest = np.ones(n, dtype=bool)
    rest[sel] = False
    piv[rk:] = np.nonzero(rest)[0]
    return piv, rk, s
