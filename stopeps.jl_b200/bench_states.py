"""Stored thermal PEPOs used as benchmark inputs.

``tfim_8x8_h3_D6_chi36_beta0.4.npz``: the beta0 = 0.4 PEPO of the 8x8 open TFIM
(J = 1, h = 3.0) prepared by this engine's ``run_purification`` path
(``src/driver/run.jl:2-43``): the identity PEPO, then ten second-order
full-update steps of tau = 0.02 at D = 6 (3+3) with exact-compression
environments at chi = 36 (18+18), FP64, no PSD repair triggered.  Made by
``python bench.py --probe purify 8 500 fp64`` on a B200 (505 s); energy per
site -2.715304489786, lnZ 87.251544694689.  Arrays: ``data`` (every site's
dense row-major block, site order x + y*Lx), ``dims`` (per site and leg the
even / odd multiplicities), ``beta``, ``log_amplitude``.
"""
from __future__ import annotations

import os

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "states")
PURIFIED_8X8 = "tfim_8x8_h3_D6_chi36_beta0.4.npz"


def load(name: str = PURIFIED_8X8):
    """(sites, dims, beta, log_amplitude) of a stored PEPO; sites in x + y*Lx order."""
    d = np.load(os.path.join(HERE, name))
    dims = np.asarray(d["dims"], np.int32)
    sites, off = [], 0
    for ld in dims:
        shape = [int(a + b) for a, b in ld]
        n = int(np.prod(shape))
        sites.append(np.asarray(d["data"][off:off + n]).reshape(shape))
        off += n
    return sites, dims, float(d["beta"]), float(d["log_amplitude"])
