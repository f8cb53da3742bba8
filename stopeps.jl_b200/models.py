"""Model and state utilities of the reference's public API.

``physical_space`` and the small-system exact diagonalisation
(``dense_hamiltonian``, ``exact_thermal_observables``,
``src/models/tfim.jl:50-76``) on the host, and ``validate_state``
(``src/states/finite.jl:53-72``) / ``identity_pepo`` (``finite.jl:80-86``)
for device states.  The ED utilities are the reference's own comparison
tools for small lattices (N <= 16); they are not on the sampling path.
"""
from __future__ import annotations

import math

import numpy as np

from .config import Lattice, TFIM


def physical_space(model: TFIM):
    """The model's physical leg (``physical_space(m)``)."""
    return model.physical_space


def dense_hamiltonian(lattice: Lattice, model: TFIM) -> np.ndarray:
    """``dense_hamiltonian`` (``tfim.jl:50-64``): H = -J sum_<ij> Z_i Z_j - h sum_i X_i on
    the open lattice, basis state b with spin i up when bit i (site x + y Lx) is 0;
    with per-site fields the X_i term carries h_i."""
    Lx, Ly = lattice.Lx, lattice.Ly
    N = Lx * Ly
    if N > 16:
        raise ValueError("ED is limited to 16 sites")
    b = np.arange(1 << N)
    spin = 1.0 - 2.0 * ((b[:, None] >> np.arange(N)[None, :]) & 1)   # (2^N, N) of +-1
    diag = np.zeros(1 << N)
    for y in range(Ly):
        for x in range(Lx):
            i = x + y * Lx
            if x + 1 < Lx:
                diag -= model.J * spin[:, i] * spin[:, i + 1]
            if y + 1 < Ly:
                diag -= model.J * spin[:, i] * spin[:, i + Lx]
    H = np.diag(diag)
    for i in range(N):
        H[b ^ (1 << i), b] -= model.field(i % Lx, i // Lx, Lx)
    return H


def exact_thermal_observables(lattice: Lattice, model: TFIM, beta: float) -> dict:
    """``exact_thermal_observables`` (``tfim.jl:71-76``): energy per site, total energy and
    log partition function at inverse temperature beta."""
    e = np.linalg.eigvalsh(dense_hamiltonian(lattice, model))
    shift = float(e.min())
    w = np.exp(-beta * (e - shift))
    Z = float(w.sum())
    total = float(w @ e / Z)
    return dict(energy_total=total, energy_per_site=total / (lattice.Lx * lattice.Ly),
                lnZ=math.log(Z) - beta * shift)


def identity_pepo(engine):
    """``identity_pepo`` (``finite.jl:80-86``): the beta = 0 thermal factor on the engine's lattice."""
    return engine.identity_pepo()


def validate_state(state):
    """``validate_state`` (``finite.jl:53-72``) of a device state: six legs per site, finite
    entries, one-dimensional auxiliary legs for a PEPS, trivial open-boundary legs and matching
    bond legs between neighbours.  Returns the state."""
    Lx, Ly = state.lattice
    sites, dims = state.download()
    dims = np.asarray(dims).reshape(Lx * Ly, -1, 2)
    peps = not state.is_pepo
    for y in range(Ly):
        for x in range(Lx):
            i = x + y * Lx
            if dims[i].shape[0] != 6:
                raise ValueError("expected six local legs")
            if not np.all(np.isfinite(sites[i])):
                raise ValueError(f"nonfinite tensor at ({x + 1},{y + 1})")
            if peps and dims[i][3].sum() != 1:
                raise ValueError("PEPS auxiliary leg must contain one irreducible carrier")
            for edge, axis in ((x == 0, 0), (y == 0, 1), (x == Lx - 1, 4), (y == Ly - 1, 5)):
                if edge and tuple(dims[i][axis]) != (1, 0):
                    raise ValueError(f"nontrivial OBC leg at ({x + 1},{y + 1})")
            if x + 1 < Lx and tuple(dims[i][4]) != tuple(dims[i + 1][0]):
                raise ValueError("horizontal space mismatch")
            if y + 1 < Ly and tuple(dims[i][5]) != tuple(dims[i + Lx][1]):
                raise ValueError("vertical space mismatch")
    return state
