"""Seeded synthetic Kohn-Sham-like orbitals for the ISDF workloads.

The reference ships only one real data set (a Si8 example, 16^3 grid). The
benchmark shapes are diamond-silicon supercells:

    Si8-like   : 1x1x1 cell, a = 10.26 bohr, 40^3 grid,  32 states
    Si64-like  : 2x2x2 cells,              80^3 grid, 256 states
    Si216-like : 3x3x3 cells,             108^3 grid, 864 states

Each state is a random combination of s / p Gaussians centred on the diamond
sites, with minimum-image distances: every site carries NEXP exponents per
orbital kind (s, px, py, pz), drawn from U[0.3, 1.5] bohr^-2, and every state
takes N(0, 1) coefficients on all of them. The states are then orthonormalised
over grid points by a Householder QR in FP64. Grid point g = ix + nx*(iy + ny*iz) sits at (ix, iy, iz) * L / n,
the layout the reference assumes (src/common/utility.cpp:711-713,
src/common/fourier.cpp:80-94). psi is returned column-major as an
(ng_total, nstate) Fortran-ordered float64 array (ld = ng_total).
"""
from __future__ import annotations

import hashlib
from dataclasses import dataclass

import numpy as np

A_SI = 10.26  # conventional cubic cell edge of diamond Si, bohr

_DIAMOND_FRAC = np.array(
    [
        [0.0, 0.0, 0.0],
        [0.0, 0.5, 0.5],
        [0.5, 0.0, 0.5],
        [0.5, 0.5, 0.0],
        [0.25, 0.25, 0.25],
        [0.25, 0.75, 0.75],
        [0.75, 0.25, 0.75],
        [0.75, 0.75, 0.25],
    ]
)


@dataclass(frozen=True)
class Shape:
    """One ISDF workload shape (one rank, S1 = S2 = all states unless set)."""

    name: str
    cells: int
    n: int  # grid points per dimension
    nstate: int
    nocc: int
    nv1: int
    nc1: int
    nv2: int
    nc2: int
    mu: int
    kmeans_iters: int = 100

    @property
    def ng(self) -> int:
        return self.n ** 3

    @property
    def length(self) -> float:
        return self.cells * A_SI


SI8 = Shape("Si8-like 40^3", 1, 40, 32, 16, 16, 16, 16, 16, 320)
SI64 = Shape("Si64-like 80^3", 2, 80, 256, 128, 128, 128, 128, 128, 2048)
SI216 = Shape("Si216-like 108^3", 3, 108, 864, 432, 432, 432, 432, 432, 4320)
# Si64's states and mu on a 40^3 grid: the profiling size (theta 1 GB, larger
# than L2, a few GB on the device in all).
SI64C = Shape("Si64-like on 40^3 (profiling)", 2, 40, 256, 128, 128, 128, 128, 128, 2048)
# Si64's grid and states with a valence x conduction pair window (S1 = the
# 128 occupied states, S2 = the 128 empty ones), the pair products a GW / BSE
# code fits; mu = 8 sqrt(128 x 128) = 1024 (the reference's default formula).
SI64VC = Shape("Si64-like valence x conduction 80^3", 2, 80, 256, 128, 128, 0, 0, 128, 1024)
# Si216's states and mu on a 40^3 grid: the profiling size of the mixed form's
# products at Si216's K and N (theta 2.2 GB).
SI216C = Shape("Si216-like on 40^3 (profiling)", 3, 40, 864, 432, 432, 432, 432, 432, 4320)
SHAPES = {"si8": SI8, "si64": SI64, "si216": SI216, "si64c": SI64C, "si216c": SI216C,
          "si64vc": SI64VC}


def diamond_sites(cells: int) -> np.ndarray:
    """Cartesian positions (bohr) of the 8*cells^3 diamond sites."""
    out = []
    for i in range(cells):
        for j in range(cells):
            for k in range(cells):
                out.append((_DIAMOND_FRAC + np.array([i, j, k])) * A_SI)
    return np.concatenate(out, axis=0)


def grid_coords(n: int, length: float) -> np.ndarray:
    """(ng, 3) coordinates, grid index g = ix + n*(iy + n*iz)."""
    h = length / n
    iz, iy, ix = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    return np.stack([ix.ravel() * h, iy.ravel() * h, iz.ravel() * h], axis=1)


NEXP = 4  # Gaussian exponents per site and orbital kind


def raw_orbitals(n: int, cells: int, nstate: int, seed: int, device: str = "cpu"):
    """Un-orthonormalised random s/p Gaussian combinations as a torch float64
    (ng, nstate) tensor on `device`. The random draws come from numpy's
    default_rng(seed), so they do not depend on the device."""
    import torch

    rng = np.random.default_rng(seed)
    length = cells * A_SI
    sites = diamond_sites(cells)
    nsite = len(sites)
    per_site = 4 * NEXP
    alphas = rng.uniform(0.3, 1.5, size=(nsite, per_site))
    coef = rng.standard_normal(size=(nsite * per_site, nstate))
    r = torch.from_numpy(grid_coords(n, length)).to(device)
    al = torch.from_numpy(alphas).to(device)
    cf = torch.from_numpy(coef).to(device)
    kind = torch.arange(per_site, device=device) % 4
    psi = torch.zeros((r.shape[0], nstate), dtype=torch.float64, device=device)
    for s in range(nsite):
        d = r - torch.from_numpy(sites[s]).to(device)
        d -= length * torch.round(d / length)  # minimum image
        d2 = (d * d).sum(dim=1, keepdim=True)
        g = torch.exp(-d2 * al[s].view(1, -1))  # (ng, per_site)
        for k in (1, 2, 3):
            g[:, kind == k] *= d[:, k - 1:k]
        psi.addmm_(g, cf[s * per_site:(s + 1) * per_site])
    return psi


def orbitals(n: int, cells: int, nstate: int, seed: int, device: str = "cpu") -> np.ndarray:
    """Orthonormal (over grid points) synthetic orbitals, (ng, nstate) F-order float64."""
    import torch

    q, _ = torch.linalg.qr(raw_orbitals(n, cells, nstate, seed, device), mode="reduced")
    return np.asfortranarray(q.cpu().numpy())


def shape_orbitals(shape: Shape, seed: int, device: str = "cpu") -> np.ndarray:
    return orbitals(shape.n, shape.cells, shape.nstate, seed, device)


def sha256(a: np.ndarray) -> str:
    return hashlib.sha256(np.asfortranarray(a).tobytes(order="F")).hexdigest()
