"""The diagonal boundary MPS on the device (``BoundaryMPSDiagonal``,
``src/contraction/diagonal_mps.jl``, ``src/sampling/diagonal_born.jl``,
``src/measurement/diagonal_energy.jl``) against the oracle's restatement
(``oracle/diagonal.py``, pinned on the CPU to the exact row contraction).

On the stored purified PEPOs (2x3 D=2, 3x3 D=4) with their truncating chi:
lognorm, the energy, <X> and the per-site <X> to 1e-10; auxiliary draws with
identical configurations and log-probabilities to 1e-9 (every truncated SVD
of the diagonal method is the full-spectrum one); the draw's conditionals
in site order; the physical kind over a projected PEPS likewise; at a chi
above every bond the device's diagonal values equal its row values; one
full-update step on diagonal bond environments against the oracle's.
"""
import numpy as np
import pytest

from util import golden, upload_golden, oracle_state, rel

pytestmark = pytest.mark.gpu
TOL = 1e-10
DRAW_TOL = 1e-9
CASES = ["pepo_2x3_D2.npz", "pepo_3x3_D4.npz"]


def _setup(sps, case):
    from oracle import diagonal as dg
    g = golden(case)
    e = sps.Engine(int(g["Lx"]), int(g["Ly"]), sps.TFIM(float(g["J"]), float(g["h"])))
    st = upload_golden(sps, g, e)
    chi, a, b = (int(v) for v in g["chi0"])
    m = sps.BoundaryMPSDiagonal(chi, None if a < 0 else sps.Z2Space(a, b))
    om = dg.BoundaryMPSDiagonal(chi, None if a < 0 else (a, b))
    return g, e, st, m, oracle_state(g), om


@pytest.mark.parametrize("case", CASES)
def test_diagonal_lognorm_and_energy(sps, case):
    from oracle import diagonal as dg, model as md
    g, e, st, m, ost, om = _setup(sps, case)
    ln, oln = sps.lognorm(st, m), dg.lognorm(ost, om)
    assert rel(ln["log_norm"], oln["log_norm"]) < TOL
    assert abs(ln["max_environment_truncation"] - oln["max_environment_truncation"]) < 1e-12
    en = sps.measure_energy(st, m, site_profile=True)
    oe = dg.measure_energy(ost, md.TFIM(float(g["J"]), float(g["h"])), om)
    for k in ("energy_per_site", "log_norm", "x_sum", "zz_sum"):
        assert rel(en[k], oe[k]) < TOL, (k, en[k], oe[k])
    np.testing.assert_allclose(en["site_x"], oe["site_x"], atol=TOL)


@pytest.mark.parametrize("case", CASES)
def test_diagonal_draws(sps, case):
    from oracle import diagonal as dg
    g, e, st, m, ost, om = _setup(sps, case)
    cache = sps.SamplingCache(st, m)
    ocache = dg.DiagonalSamplingCache(ost, om)
    Lx, Ly = int(g["Lx"]), int(g["Ly"])
    order = dg.draw_order(Lx, Ly)
    for u in g["uniforms"][:3]:
        d = sps.sample_conditionals(cache, uniforms=u)
        od = dg.sample_configuration(ocache, uniforms=u)
        np.testing.assert_array_equal(d["configuration"], np.asarray(od["configuration"]))
        again = sps.sample_configuration(cache, configuration=d["configuration"])
        assert rel(again["log_probability"], od["log_probability"]) < DRAW_TOL
        for i, (x, y) in enumerate(order):   # conditionals come back in site order
            assert abs(d["conditionals"][x, y] - od["conditionals"][i]) < DRAW_TOL


def test_diagonal_physical_draws(sps):
    from oracle import diagonal as dg, sampling as osp
    g, e, st, m, ost, om = _setup(sps, "pepo_3x3_D4.npz")
    cfg = np.asarray(g["configs"][0])
    ps, _ = sps.project_configuration(st, cfg)
    ops, _ = osp.project_configuration(ost, cfg.tolist())
    cache = sps.SamplingCache(ps, m, kind="physical")
    ocache = dg.DiagonalSamplingCache(ops, om, kind="physical")
    for seed in range(2):
        u = np.random.default_rng([17, seed]).random(9)
        d = sps.sample_configuration(cache, uniforms=u)
        od = dg.sample_configuration(ocache, uniforms=u)
        np.testing.assert_array_equal(d["configuration"], np.asarray(od["configuration"]))
        assert rel(d["log_probability"], od["log_probability"]) < DRAW_TOL
        zero = sum(1 for r in od["repairs"] if r.get("reason") == "zero_proposal_weights")
        assert d["zero_proposals"] == zero


def test_diagonal_exact_chi_equals_row_contraction(sps):
    """2x3 D=2 at chi = 64 (above every bond): both device contractions are exact."""
    g = golden("pepo_2x3_D2.npz")
    e = sps.Engine(2, 3, sps.TFIM(float(g["J"]), float(g["h"])))
    st = upload_golden(sps, g, e)
    a = sps.measure_energy(st, sps.BoundaryMPS(64))
    b = sps.measure_energy(st, sps.BoundaryMPSDiagonal(64))
    for k in ("energy_per_site", "log_norm", "x_sum"):
        assert rel(a[k], b[k]) < 1e-12, k
    ca, cb = sps.SamplingCache(st, sps.BoundaryMPS(64)), sps.SamplingCache(st, sps.BoundaryMPSDiagonal(64))
    cfgs = np.stack([np.asarray(c) for c in g["configs"][:3]])
    la, _ = sps.sample_probability_batch(ca, cfgs)
    lb, _ = sps.sample_probability_batch(cb, cfgs)
    np.testing.assert_allclose(lb, la, rtol=1e-12)


@pytest.mark.parametrize("case", CASES)
def test_diagonal_full_update_step(sps, case):
    """One second-order full-update step of the projected PEPS on diagonal
    bond environments (``diagonal_update.jl``) against the oracle's step:
    bond count, stop reasons, the log normalisation and the stepped state's
    energy and lnZ to 1e-9 (the row step's tolerance)."""
    from oracle import diagonal as dg, full_update as fu, model as md, sampling as osp
    g = golden(case)
    upd = sps.FullUpdate(max_iterations=8, linear_max_iterations=40) if "2x3" in case else sps.FullUpdate()
    e = sps.Engine(int(g["Lx"]), int(g["Ly"]), sps.TFIM(float(g["J"]), float(g["h"])), update=upd)
    st = upload_golden(sps, g, e)
    pc = g["peps_cfg"]
    chi, a, b = int(pc[3]), int(pc[4]), int(pc[5])
    m = sps.BoundaryMPSDiagonal(chi, None if a < 0 else sps.Z2Space(a, b))
    om = dg.BoundaryMPSDiagonal(chi, None if a < 0 else (a, b))
    space = None if pc[1] < 0 else (int(pc[1]), int(pc[2]))
    cfg = np.asarray(g["configs"][0])
    ps, _ = sps.project_configuration(st, cfg)
    ops, _ = osp.project_configuration(oracle_state(g), cfg.tolist())
    r = sps.evolution_step(ps, float(g["dtau"]), int(pc[0]), m, None if space is None else sps.Z2Space(*space))
    opts = fu.FullUpdate(upd.max_iterations, upd.error_tolerance, upd.diagonal_shift, upd.linear_max_iterations,
                         upd.linear_tolerance)
    model = md.TFIM(float(g["J"]), float(g["h"]))
    orr = fu.evolution_step(ops, model, float(g["dtau"]), int(pc[0]), opts, om, space=space)
    assert r["bond_updates"] == orr["bond_updates"]
    stops = [r["stop_error_tolerance"], r["stop_iteration_limit"], r["stop_residual_fallback"], r["stop_disabled"]]
    assert stops == [orr["stop_reasons"][k] for k in ("error_tolerance", "iteration_limit", "residual_fallback",
                                                       "disabled")]
    assert rel(r["log_normalization_sum"], sum(v for _, v in orr["normalizations"])) < 1e-9
    en = sps.measure_energy(ps, m)
    oe = dg.measure_energy(ops, model, om)
    assert rel(en["energy_per_site"], oe["energy_per_site"]) < 1e-9
    assert rel(en["log_norm"], oe["log_norm"]) < 1e-9


def test_diagonal_forced_psd_repair_matches_oracle(sps):
    """update_bond!'s PSD-repair branch forced on every bond of one step on
    diagonal bond environments: the repaired metric from the diagonal bond
    hole and the refit, against the oracle with the same bonds forced."""
    from oracle import diagonal as dg, full_update as fu, model as md, sampling as osp
    g = golden("pepo_2x3_D2.npz")
    upd = sps.FullUpdate(max_iterations=8, linear_max_iterations=40)
    e = sps.Engine(2, 3, sps.TFIM(float(g["J"]), float(g["h"])), update=upd)
    st = upload_golden(sps, g, e)
    pc = g["peps_cfg"]
    chi = int(pc[3])
    m = sps.BoundaryMPSDiagonal(chi, None)
    cfg = g["configs"][0]
    ps, _ = sps.project_configuration(st, cfg)
    e.set_injection(force_repair=True)
    try:
        r = sps.evolution_step(ps, float(g["dtau"]), int(pc[0]), m, None)
    finally:
        e.set_injection()
    assert r["repairs"] == r["bond_updates"] > 0
    ops, _ = osp.project_configuration(oracle_state(g), np.asarray(cfg).tolist())
    bonds = {((0, y), (1, y)) for y in range(3)} | {((x, y), (x, y + 1)) for x in range(2) for y in range(2)}
    model = md.TFIM(float(g["J"]), float(g["h"]))
    ro = fu.evolution_step(ops, model, float(g["dtau"]), int(pc[0]), fu.FullUpdate(max_iterations=8,
                           linear_max_iterations=40), dg.BoundaryMPSDiagonal(chi), force_repair_bonds=bonds)
    assert ro["repairs"] == r["repairs"]
    assert rel(r["log_normalization_sum"], sum(v for _, v in ro["normalizations"])) < 1e-9
    en = sps.measure_energy(ps, m)
    oen = dg.measure_energy(ops, model, dg.BoundaryMPSDiagonal(chi))
    assert rel(en["energy_per_site"], oen["energy_per_site"]) < 1e-9


@pytest.mark.parametrize("contraction", ["BoundaryMPSDiagonal", "BoundaryMPSDiagonalVariational"])
def test_pipeline_on_diagonal_boundaries_matches_the_oracle_ops(sps, contraction):
    """``RunConfig(contraction=...)`` end to end on the device (purification on
    diagonal bond environments, diagonal draws, projection, evolution and
    measurement) against the same driver with the oracle as the numerical
    ops: the same draws and the same curve."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from test_parallel import OracleOps
    c = sps.RunConfig(lattice=sps.Lattice(2, 3), model=sps.TFIM(1.0, 0.7), beta0=0.1, beta_log=[0.1, 0.2],
                      beta_measure=[0.1, 0.2], delta_tau_pur=0.05, delta_tau_peps=0.05, D_pur=2, D_peps=2,
                      chi_environment=4, Ns=4, seed=3, contraction=getattr(sps, contraction),
                      resampling=sps.ResamplingOptions(enabled=False))
    dev = sps.run_stochastic(c, sps.run_purification(c))
    ops = OracleOps(c)
    ref = sps.run_stochastic(c, sps.run_purification(c, ops=ops, identity=ops.identity), ops=ops)
    for d, o in zip(dev["diagnostics"]["born_draws"], ref["diagnostics"]["born_draws"]):
        np.testing.assert_array_equal(d["configuration"], o["configuration"])
        assert rel(d["log_probability"], o["log_probability"]) < 1e-9
    curve = [r for r in dev["observables"]["curve"] if r.get("source") == "sampling"]
    ocurve = [r for r in ref["observables"]["curve"] if r.get("source") == "sampling"]
    assert len(curve) == len(ocurve) > 0
    for a, b in zip(curve, ocurve):
        assert rel(a["lnZ"], b["lnZ"]) < 1e-9
        assert (np.isnan(a["energy_per_site"]) and np.isnan(b["energy_per_site"])) or \
            rel(a["energy_per_site"], b["energy_per_site"]) < 1e-9
