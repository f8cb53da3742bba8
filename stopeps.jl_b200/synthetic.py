"""Seeded synthetic thermal PEPOs with the shapes of the benchmark workloads.

The reference prepares its beta0 PEPO by purification (``run_purification``);
for throughput measurements a seeded stand-in with the same lattice, bond
sectors and tensor layout is used: the identity thermal factor of
``identity_pepo`` (``src/states/finite.jl:80-86``) embedded in Z2 bonds of
dimension D = D/2 + D/2, plus ``eps`` times Gaussian noise on every Z2-allowed
entry, normalised per site.  Its contraction cost is that of a purified
PEPO with the same D; its spectrum is closer to a product state.
"""
from __future__ import annotations

import numpy as np


def z2_mask(dims):
    """Boolean mask of even-parity entries for legs given as (n0, n1)."""
    par = [np.concatenate([np.zeros(a, np.int64), np.ones(b, np.int64)]) for a, b in dims]
    tot = np.zeros([a + b for a, b in dims], np.int64)
    for k, p in enumerate(par):
        sh = [1] * len(dims)
        sh[k] = len(p)
        tot = tot + p.reshape(sh)
    return tot % 2 == 0


def synthetic_pepo(Lx: int, Ly: int, D: int, eps: float = 0.15, seed: int = 7):
    """Site tensors (x + y*Lx order) and per-leg (n0, n1) of the stand-in PEPO."""
    if D % 2:
        raise ValueError("D must be even (D/2 + D/2 sectors)")
    rng = np.random.default_rng(seed)
    h = D // 2
    sites, dims = [], []
    for y in range(Ly):
        for x in range(Lx):
            ld = [(1, 0) if x == 0 else (h, h), (1, 0) if y == 0 else (h, h), (1, 1), (1, 1),
                  (1, 0) if x == Lx - 1 else (h, h), (1, 0) if y == Ly - 1 else (h, h)]
            shape = [a + b for a, b in ld]
            a = rng.standard_normal(shape) * eps * z2_mask(ld)
            a[0, 0, 0, 0, 0, 0] += 1.0
            a[0, 0, 1, 1, 0, 0] += 1.0
            a /= np.sqrt(np.sum(a * a))
            sites.append(a)
            dims.append(ld)
    return sites, np.asarray(dims, np.int32)
