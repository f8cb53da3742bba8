"""Shared helpers of the test suite (fixture loading, oracle <-> device states)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def space(a, b):
    return None if a < 0 else (int(a), int(b))


def upload_golden(sps, g, engine):
    """Upload the fixture PEPO into ``engine``."""
    L = int(g["Lx"]) * int(g["Ly"])
    dims = g["dims"].reshape(L, 6, 2)
    sites, off = [], 0
    for i in range(L):
        n = int(np.prod([a + b for a, b in dims[i]]))
        sites.append(g["data"][off:off + n])
        off += n
    return engine.upload_state(sites, dims, True, beta=float(g["beta"]), log_amplitude=float(g["log_amplitude"]))


def oracle_state(g):
    """The fixture PEPO as an oracle state."""
    from oracle.model import State
    from oracle.z2 import T, leg
    Lx, Ly = int(g["Lx"]), int(g["Ly"])
    dims = g["dims"].reshape(Lx * Ly, 6, 2)
    sites = [[None] * Ly for _ in range(Lx)]
    off = 0
    for i in range(Lx * Ly):
        shape = [int(a + b) for a, b in dims[i]]
        n = int(np.prod(shape))
        x, y = i % Lx, i // Lx
        sites[x][y] = T(g["data"][off:off + n].reshape(shape), [leg(int(a), int(b)) for a, b in dims[i]])
        off += n
    return State(Lx, Ly, sites, float(g["beta"]), float(g["log_amplitude"]), "pepo")


def rel(a, b):
    return abs(a - b) / max(1.0, abs(b))
