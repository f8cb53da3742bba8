"""The row variational boundary MPS on the device (``BoundaryMPSRowVariational``,
``src/contraction/row_variational.jl``) against the oracle's restatement
(``oracle/variational.py``, pinned on the CPU to the exact contraction).

The sweep count is fixed (``threshold_sweep = 0``, three round trips) so that
rounding cannot move a stopping decision; lognorm, the energy, <X> and the
Born draws then agree to 1e-10 (draws 1e-9) on the stored purified PEPOs at
their truncating chi, and the fit summary matches; likewise the diagonal
variational method (``src/contraction/diagonal_variational.jl``) against
``oracle/diagonal_variational.py``.
"""
import numpy as np
import pytest

from util import golden, upload_golden, oracle_state, rel

pytestmark = pytest.mark.gpu
TOL = 1e-10
CASES = ["pepo_2x3_D2.npz", "pepo_3x3_D4.npz"]


def _setup(sps, case):
    from oracle import variational as va
    g = golden(case)
    e = sps.Engine(int(g["Lx"]), int(g["Ly"]), sps.TFIM(float(g["J"]), float(g["h"])))
    st = upload_golden(sps, g, e)
    chi, a, b = (int(v) for v in g["chi0"])
    m = sps.BoundaryMPSRowVariational(chi, None if a < 0 else sps.Z2Space(a, b), max_sweep=3, threshold_sweep=0.0)
    om = va.BoundaryMPSRowVariational(chi, None if a < 0 else (a, b), max_sweep=3, threshold_sweep=0.0)
    return g, e, st, m, oracle_state(g), om


@pytest.mark.parametrize("case", CASES)
def test_variational_lognorm_energy_and_draws(sps, case):
    from oracle import boundary as bm, model as md, sampling as osp
    g, e, st, m, ost, om = _setup(sps, case)
    ln, oln = sps.lognorm(st, m), bm.lognorm(ost, om)
    assert rel(ln["log_norm"], oln["log_norm"]) < TOL
    assert ln["boundary_variational"]["layers"] == len(oln["boundary_variational"]["layers"])
    assert ln["boundary_variational"]["max_sweeps"] == oln["boundary_variational"]["max_sweeps"]
    assert ln["boundary_variational"]["fallback_count"] == oln["boundary_variational"]["fallback_count"]
    en = sps.measure_energy(st, m)
    oe = osp.measure_energy(ost, md.TFIM(float(g["J"]), float(g["h"])), om)
    for k in ("energy_per_site", "log_norm", "x_sum"):
        assert rel(en[k], oe[k]) < TOL, (k, en[k], oe[k])
    cache, ocache = sps.SamplingCache(st, m), osp.SamplingCache(ost, om)
    for u in g["uniforms"][:2]:
        d = sps.sample_configuration(cache, uniforms=u)
        od = osp.sample_configuration(ocache, uniforms=u)
        np.testing.assert_array_equal(d["configuration"], np.asarray(od["configuration"]))
        assert rel(d["log_probability"], od["log_probability"]) < 1e-9


def test_variational_options_are_checked(sps):
    g, e, st, m, ost, om = _setup(sps, "pepo_2x3_D2.npz")
    with pytest.raises(sps._lib.EngineError):
        e.check(e.lib.sps_set_variational(e.h, 0, 1e-8))
    with pytest.raises(ValueError):
        sps.BoundaryMPSRowVariational(4, None, max_sweep=0)


@pytest.mark.parametrize("case", CASES)
def test_diagonal_variational_lognorm_energy_and_draws(sps, case):
    """``BoundaryMPSDiagonalVariational`` (``diagonal_variational.jl``) against the
    oracle's restatement with two fixed round trips per layer."""
    from oracle import diagonal as dg, diagonal_variational as dv, model as md
    g = golden(case)
    e = sps.Engine(int(g["Lx"]), int(g["Ly"]), sps.TFIM(float(g["J"]), float(g["h"])))
    st = upload_golden(sps, g, e)
    ost = oracle_state(g)
    chi, a, b = (int(v) for v in g["chi0"])
    m = sps.BoundaryMPSDiagonalVariational(chi, None if a < 0 else sps.Z2Space(a, b), max_sweep=2,
                                           threshold_sweep=0.0)
    om = dv.BoundaryMPSDiagonalVariational(chi, None if a < 0 else (a, b), max_sweep=2, threshold_sweep=0.0)
    ln, oln = sps.lognorm(st, m), dg.lognorm(ost, om)
    assert rel(ln["log_norm"], oln["log_norm"]) < TOL
    assert ln["boundary_variational"]["layers"] == len(oln["boundary_variational"]["layers"])
    assert ln["boundary_variational"]["fallback_count"] == oln["boundary_variational"]["fallback_count"]
    en = sps.measure_energy(st, m)
    oe = dg.measure_energy(ost, md.TFIM(float(g["J"]), float(g["h"])), om)
    for k in ("energy_per_site", "log_norm", "x_sum"):
        assert rel(en[k], oe[k]) < TOL, (k, en[k], oe[k])
    cache, ocache = sps.SamplingCache(st, m), dg.DiagonalSamplingCache(ost, om)
    for u in g["uniforms"][:2]:
        d = sps.sample_configuration(cache, uniforms=u)
        od = dg.sample_configuration(ocache, uniforms=u)
        np.testing.assert_array_equal(d["configuration"], np.asarray(od["configuration"]))
        assert rel(d["log_probability"], od["log_probability"]) < 1e-9


def test_pipeline_on_row_variational_boundaries_matches_the_oracle_ops(sps):
    """``RunConfig(contraction=BoundaryMPSRowVariational)`` end to end on the
    device against the same driver with the oracle as the numerical ops."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from test_parallel import OracleOps
    c = sps.RunConfig(lattice=sps.Lattice(3, 2), model=sps.TFIM(1.0, 0.7), beta0=0.1, beta_log=[0.1, 0.2],
                      beta_measure=[0.1, 0.2], delta_tau_pur=0.05, delta_tau_peps=0.05, D_pur=2, D_peps=2,
                      chi_environment=4, Ns=4, seed=3, contraction=sps.BoundaryMPSRowVariational,
                      resampling=sps.ResamplingOptions(enabled=False))
    dev = sps.run_stochastic(c, sps.run_purification(c))
    ops = OracleOps(c)
    ref = sps.run_stochastic(c, sps.run_purification(c, ops=ops, identity=ops.identity), ops=ops)
    for d, o in zip(dev["diagnostics"]["born_draws"], ref["diagnostics"]["born_draws"]):
        np.testing.assert_array_equal(d["configuration"], o["configuration"])
        assert rel(d["log_probability"], o["log_probability"]) < 1e-9
    for a, b in zip([r for r in dev["observables"]["curve"] if r.get("source") == "sampling"],
                    [r for r in ref["observables"]["curve"] if r.get("source") == "sampling"]):
        assert rel(a["lnZ"], b["lnZ"]) < 1e-9
        assert rel(a["energy_per_site"], b["energy_per_site"]) < 1e-9
