"""TFIM model, finite states and exact diagonalization for the CPU oracle.

TEST INFRASTRUCTURE ONLY (see ``oracle/z2.py``).

Restates ``src/models/tfim.jl`` and ``src/states/finite.jl`` for the Z2
symmetric TFIM (``TFIM(physical_space=Z2Space(0=>1,1=>1))``): basis state 0 is
the even parity state |+x>, state 1 the odd state |-x>, so X is diagonal and
Z flips parity.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .z2 import T, leg, norm

P2 = leg(1, 1)       # physical / auxiliary leg Z2Space(0=>1,1=>1)
TRIV = leg(1, 0)     # open-boundary unit leg


@dataclass
class TFIM:
    """``TFIM(J,h)`` with Z2 physical space (``src/models/tfim.jl:9-19``).

    ``fields`` (optional, Lx*Ly values in x + y*Lx order) replaces the uniform
    h by a field per site: the extension a per-site gradient needs (the
    reference's model has one h).  The bond gates then split each site's own
    field over its bonds (h_i / deg_i, as ``tfim.jl:46`` does with h)."""
    J: float = 1.0
    h: float = 0.7
    fields: tuple | None = None

    def field(self, x, y, Lx):
        """The transverse field at 0-based site (x, y)."""
        return self.h if self.fields is None else float(self.fields[x + y * Lx])


def spin_operators():
    """X (parity-diagonal) and the two-site ZZ (``src/models/tfim.jl:22-34``)."""
    X = np.diag([1.0, -1.0])
    z = np.array([[0.0, 1.0], [1.0, 0.0]])
    ZZ = np.einsum("pu,qv->pquv", z, z)
    return X, z, ZZ


def degree(Lx, Ly, x, y):
    """Number of lattice neighbours (``src/models/tfim.jl:42``), 0-based site."""
    return (x > 0) + (x < Lx - 1) + (y > 0) + (y < Ly - 1)


def bond_hamiltonian(m: TFIM, Lx, Ly, a, b):
    """-J ZZ - h/deg(a) X(x)I - h/deg(b) I(x)X as H[p,q,u,v] (``tfim.jl:44-47``)."""
    X, z, ZZ = spin_operators()
    I = np.eye(2)
    da = degree(Lx, Ly, *a)
    db = degree(Lx, Ly, *b)
    ha, hb = m.field(*a, Lx), m.field(*b, Lx)
    return (-m.J * ZZ - (ha / da) * np.einsum("pu,qv->pquv", X, I)
            - (hb / db) * np.einsum("pu,qv->pquv", I, X))


def sym_expm(Hm: np.ndarray, t: float) -> np.ndarray:
    """exp(t*H) of a real symmetric matrix through its eigendecomposition."""
    w, V = np.linalg.eigh(0.5 * (Hm + Hm.T))
    return (V * np.exp(t * w)) @ V.T


def trotter_gate(m: TFIM, Lx, Ly, a, b, delta) -> T:
    """exp(-delta * h_bond) as a 4-leg tensor gate[p,q,u,v] (``tfim.jl:48``)."""
    H = bond_hamiltonian(m, Lx, Ly, a, b).reshape(4, 4)
    G = sym_expm(H, -delta).reshape(2, 2, 2, 2)
    return T(G, [P2, P2, P2, P2])


def onsite_gate(m: TFIM, delta) -> np.ndarray:
    """The one-site lattice's gate exp(delta h X) (the site's own field)."""
    X, _, _ = spin_operators()
    return sym_expm(-m.field(0, 0, 1) * X, -delta)


@dataclass
class State:
    """``FiniteState``: sites[x][y] with legs (W,N,Pout,Paux,E,S)."""
    Lx: int
    Ly: int
    sites: list
    beta: float = 0.0
    log_amplitude: float = 0.0
    kind: str = "pepo"

    def copy(self) -> "State":
        return State(self.Lx, self.Ly, [[s.copy() for s in col] for col in self.sites],
                     self.beta, self.log_amplitude, self.kind)

    def __getitem__(self, xy):
        return self.sites[xy[0]][xy[1]]

    def __setitem__(self, xy, v):
        self.sites[xy[0]][xy[1]] = v


def site_order(Lx, Ly):
    """Row-major traversal, x fastest (``src/states/finite.jl:10``)."""
    return [(x, y) for y in range(Ly) for x in range(Lx)]


def identity_pepo(Lx, Ly) -> State:
    """Identity thermal factor at beta=0 (``src/states/finite.jl:80-86``)."""
    a = np.zeros((1, 1, 2, 2, 1, 1))
    a[0, 0, 0, 0, 0, 0] = 1.0
    a[0, 0, 1, 1, 0, 0] = 1.0
    sites = [[T(a, [TRIV, TRIV, P2, P2, TRIV, TRIV]) for _ in range(Ly)] for _ in range(Lx)]
    return State(Lx, Ly, sites, 0.0, 0.0, "pepo")


def normalize_state(s: State):
    """Per-site Frobenius normalisation in row-major order (``finite.jl:89-100``)."""
    records = []
    for (x, y) in site_order(s.Lx, s.Ly):
        v = norm(s[x, y])
        if not (math.isfinite(v) and v > 0):
            raise RuntimeError(f"zero or nonfinite tensor at {(x + 1, y + 1)}")
        s[x, y] = s[x, y] / v
        inc = math.log(v)
        s.log_amplitude += inc
        records.append(((x + 1, y + 1), inc))
    return records


# ---------------------------------------------------------------------------
# exact diagonalization (src/models/tfim.jl:50-76)
# ---------------------------------------------------------------------------

def dense_hamiltonian(Lx, Ly, m: TFIM) -> np.ndarray:
    N = Lx * Ly
    if N > 16:
        raise ValueError("ED is limited to 16 sites")
    dim = 1 << N
    b = np.arange(dim)
    H = np.zeros((dim, dim))

    def idx(x, y):
        return x + y * Lx

    def z(i):
        return np.where((b >> i) & 1, -1.0, 1.0)

    diag = np.zeros(dim)
    for y in range(Ly):
        for x in range(Lx - 1):
            diag -= m.J * z(idx(x, y)) * z(idx(x + 1, y))
    for y in range(Ly - 1):
        for x in range(Lx):
            diag -= m.J * z(idx(x, y)) * z(idx(x, y + 1))
    H[b, b] = diag
    for i in range(N):
        H[b ^ (1 << i), b] -= m.field(i % Lx, i // Lx, Lx)
    return H


def exact_thermal_observables(Lx, Ly, m: TFIM, beta: float):
    e = np.linalg.eigvalsh(dense_hamiltonian(Lx, Ly, m))
    shift = e.min()
    w = np.exp(-beta * (e - shift))
    Z = w.sum()
    total = float(w @ e / Z)
    return dict(energy_total=total, energy_per_site=total / (Lx * Ly),
                lnZ=float(math.log(Z) - beta * shift))


def exact_thermal_magnetization(Lx, Ly, m: TFIM, beta: float) -> float:
    """<sum_i X_i>/N at inverse temperature beta by ED (extension; no reference API)."""
    H = dense_hamiltonian(Lx, Ly, m)
    e, V = np.linalg.eigh(H)
    N = Lx * Ly
    dim = 1 << N
    b = np.arange(dim)
    Xsum = np.zeros((dim, dim))
    for i in range(N):
        Xsum[b ^ (1 << i), b] += 1.0
    w = np.exp(-beta * (e - e.min()))
    xs = np.einsum("ik,ij,jk->k", V, Xsum, V)
    return float((w @ xs) / w.sum() / N)
