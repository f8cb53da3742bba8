"""Per-site transverse fields h_i on the device (an extension of the reference's
TFIM, which has one h: ``src/models/tfim.jl:9-19``), against the oracle's
restatement of the same model (``oracle/model.py``), which is pinned to exact
diagonalisation with second-order Trotter convergence on the CPU.

A fresh purification to beta = 0.2 on a 3x2 lattice with D = 3 and a
truncating boundary (chi = 6): lnZ, energy and <X> agree at 1e-9 relative, as
in the uniform-field live test.  Fields that repeat the uniform h give the
uniform run's values: the gates are the same numbers, only the energy's field
sum runs site by site.
"""
import numpy as np
import pytest

from util import rel

pytestmark = pytest.mark.gpu
TOL = 1e-9


def _kw():
    return dict(beta0=0.1, beta_log=[0.1], beta_measure=[0.1], delta_tau_pur=0.05, D_pur=3, D_peps=3,
                chi_environment=6, Ns=1)


def test_per_site_fields_match_oracle(sps):
    from oracle import driver as odr
    f = tuple(1.3 + np.random.default_rng(11).uniform(-0.4, 0.4, 6))
    c = sps.RunConfig(lattice=sps.Lattice(3, 2), model=sps.TFIM(1.0, 1.3, fields=f), **_kw(),
                      resampling=sps.ResamplingOptions(enabled=False))
    oc = odr.RunConfig(Lx=3, Ly=2, J=1.0, h=1.3, fields=f, **_kw())
    cp = sps.run_purification(c)
    _, rows = odr.run_purification(oc)
    assert len(cp.purification) == len(rows)
    for a, b in zip(cp.purification, rows):
        for k in ("lnZ", "energy_per_site", "magnetization"):
            assert (np.isnan(a[k]) and np.isnan(b[k])) or rel(a[k], b[k]) < TOL, (k, a[k], b[k])


def test_uniform_fields_written_per_site(sps):
    kw = dict(lattice=sps.Lattice(3, 2), **_kw(), resampling=sps.ResamplingOptions(enabled=False))
    a = sps.run_purification(sps.RunConfig(model=sps.TFIM(1.0, 1.3), **kw)).purification[-1]
    b = sps.run_purification(sps.RunConfig(model=sps.TFIM(1.0, 1.3, fields=[1.3] * 6), **kw)).purification[-1]
    # two runs of the full update: its iterative solves may carry run-to-run
    # rounding, so the bar is the parity one
    assert rel(a["lnZ"], b["lnZ"]) < 1e-10
    assert rel(a["energy_per_site"], b["energy_per_site"]) < 1e-10


def test_pipeline_with_site_fields_matches_the_oracle_ops(sps):
    """run_stochastic with per-site fields on the device against the same
    driver with the oracle as the numerical ops."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from test_parallel import OracleOps
    f = (0.5, 0.9, 0.7, 1.1, 0.6, 1.3)
    c = sps.RunConfig(lattice=sps.Lattice(3, 2), model=sps.TFIM(1.0, 0.7, fields=f), beta0=0.1,
                      beta_log=[0.1, 0.2], beta_measure=[0.1, 0.2], delta_tau_pur=0.05, delta_tau_peps=0.05,
                      D_pur=2, D_peps=2, chi_environment=4, Ns=4, seed=3,
                      resampling=sps.ResamplingOptions(enabled=False))
    dev = sps.run_stochastic(c, sps.run_purification(c))
    ops = OracleOps(c)
    ref = sps.run_stochastic(c, sps.run_purification(c, ops=ops, identity=ops.identity), ops=ops)
    for a, b in zip([r for r in dev["observables"]["curve"] if r.get("source") == "sampling"],
                    [r for r in ref["observables"]["curve"] if r.get("source") == "sampling"]):
        assert rel(a["lnZ"], b["lnZ"]) < 1e-9
        assert rel(a["energy_per_site"], b["energy_per_site"]) < 1e-9
