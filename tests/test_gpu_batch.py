"""Batched C-ABI variants and host-side failure injection, on the GPU.

``sps_project_batch``, ``sps_measure_energy_batch``, ``sps_lognorm_batch`` and
``sps_evolution_step_batch`` replace the reference's per-particle loops
(``src/driver/run.jl:52-57``, ``:104-108``); with several samples at the same
time (own stream and workspace each) they must give the single-sample
results.  The injection tests reach the library's error paths from the host
(a forced PSD repair, a Jacobi sweep cap, a Born conditional with zero total
mass); nothing faults on the device.
"""
import numpy as np
import pytest

from util import golden, upload_golden, oracle_state, rel

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _engine(sps, g, **kw):
    return sps.Engine(int(g["Lx"]), int(g["Ly"]), sps.TFIM(float(g["J"]), float(g["h"])), **kw)


def _env(sps, g):
    pc = g["peps_cfg"]
    m = sps.BoundaryMPS(int(pc[3]), None if pc[4] < 0 else sps.Z2Space(int(pc[4]), int(pc[5])))
    sp = None if pc[1] < 0 else sps.Z2Space(int(pc[1]), int(pc[2]))
    return int(pc[0]), m, sp


@pytest.mark.parametrize("case", ["pepo_3x3_D4.npz", "pepo_4x4_D4.npz"])
def test_batch_entry_points_match_single_calls(sps, case):
    g = golden(case)
    e = _engine(sps, g)
    st = upload_golden(sps, g, e)
    D, m, sp = _env(sps, g)
    cfgs = np.asarray(g["configs"])
    single = [sps.project_configuration(st, c) for c in cfgs]
    e.set_concurrency(3)
    try:
        states, lns = sps.project_batch(st, cfgs)
        for (s1, n1), s2, n2 in zip(single, states, lns):
            np.testing.assert_allclose(n2, n1, rtol=1e-13, atol=1e-13)
        en_b = sps.measure_energy_batch(states, m)
        ln_b = sps.lognorm_batch(states, m)
        dt = float(g["dtau"])
        reps_b = sps.evolution_step_batch(states, [dt] * len(states), D, m, sp)
        en_after_b = sps.measure_energy_batch(states, m)
    finally:
        e.set_concurrency(1)
    for (s1, _), eb, lb, rb, eab in zip(single, en_b, ln_b, reps_b, en_after_b):
        e1 = sps.measure_energy(s1, m)
        assert rel(eb["energy_per_site"], e1["energy_per_site"]) < 1e-12
        assert rel(eb["x_sum"], e1["x_sum"]) < 1e-12
        l1 = sps.lognorm(s1, m)
        assert rel(lb["log_norm"], l1["log_norm"]) < 1e-12
        r1 = sps.evolution_step(s1, float(g["dtau"]), D, m, sp)
        assert rb["bond_updates"] == r1["bond_updates"]
        assert rel(rb["log_normalization_sum"], r1["log_normalization_sum"]) < 1e-11
        ea1 = sps.measure_energy(s1, m)
        assert rel(eab["energy_per_site"], ea1["energy_per_site"]) < 1e-11
    # the first projected sample against the oracle fixture (evolution step included)
    assert rel(en_after_b[0]["energy_per_site"], float(g["step_energy"][0])) < 1e-9


def test_batch_rejects_a_state_twice(sps):
    g = golden("pepo_3x3_D4.npz")
    e = _engine(sps, g)
    st = upload_golden(sps, g, e)
    D, m, sp = _env(sps, g)
    ps, _ = sps.project_configuration(st, g["configs"][0])
    with pytest.raises(sps._lib.EngineError):
        sps.measure_energy_batch([ps, ps], m)


def test_run_stochastic_uses_the_batched_calls(sps):
    """run_stochastic with concurrency > 1 (every phase batched) reproduces the
    serial run's draws, weights and curve."""
    kw = dict(lattice=sps.Lattice(2, 2), model=sps.TFIM(1.0, 0.7), beta0=0.2, beta_log=[0.1, 0.2, 0.3],
              beta_measure=[0.2, 0.3], delta_tau_pur=0.05, delta_tau_peps=0.05, D_pur=2, D_peps=2,
              bond_space_pur=sps.Z2Space(1, 1), bond_space_peps=sps.Z2Space(1, 1), chi_environment=4,
              environment_space=sps.Z2Space(2, 2), Ns=6, seed=3, resampling=sps.ResamplingOptions(enabled=False))
    c = sps.RunConfig(**kw)
    g = golden("pipeline_2x2.npz")
    cp = sps.run_purification(c)
    cp.state.engine.set_concurrency(4)
    try:
        res = sps.run_stochastic(c, cp)
    finally:
        cp.state.engine.set_concurrency(1)
    draws = res["diagnostics"]["born_draws"]
    np.testing.assert_array_equal(np.stack([d["configuration"] for d in draws]), g["draw_cfg"])
    curve = [r for r in res["observables"]["curve"] if r.get("source") == "sampling"]
    np.testing.assert_allclose([r["energy_per_site"] for r in curve], g["energy"], rtol=1e-10)
    np.testing.assert_allclose([r["lnZ"] for r in curve], g["lnZ"], rtol=1e-10)
    np.testing.assert_allclose([r["eta"] for r in curve], g["eta"], rtol=1e-10)


@pytest.mark.parametrize("multi_cta", [False, True])
def test_forced_psd_repair_matches_oracle(sps, multi_cta):
    """update_bond!'s PSD-repair branch (full_update.jl:490-501) forced on
    every bond of one step: the repaired metric (hole in the (bras | kets)
    grouping, per-sector eigendecomposition, negative eigenvalues clipped) and
    the refit, against the oracle with the same bonds forced.  multi_cta: the
    parity blocks of 32 rows and more take the multi-CTA route of large holes
    (one-sided Jacobi of the shifted hole) at this small size."""
    from oracle import full_update as fu, model as md, boundary as bm, sampling as osp
    g = golden("pepo_2x3_D2.npz")
    upd = sps.FullUpdate(max_iterations=8, linear_max_iterations=40)
    e = _engine(sps, g, update=upd)
    st = upload_golden(sps, g, e)
    D, m, sp = _env(sps, g)
    cfg = g["configs"][0]
    ps, _ = sps.project_configuration(st, cfg)
    e.set_injection(force_repair=True, multi_cta_eigh_min=32 if multi_cta else 0)
    try:
        r = sps.evolution_step(ps, float(g["dtau"]), D, m, sp)
    finally:
        e.set_injection()
    assert r["repairs"] == r["bond_updates"] > 0
    ost = oracle_state(g)
    ops, _ = osp.project_configuration(ost, np.asarray(cfg).tolist())
    Lx, Ly = int(g["Lx"]), int(g["Ly"])
    bonds = {((x, y), (x + 1, y)) for x in range(Lx - 1) for y in range(Ly)}
    bonds |= {((x, y), (x, y + 1)) for x in range(Lx) for y in range(Ly - 1)}
    pc = g["peps_cfg"]
    om = bm.BoundaryMPS(int(pc[3]), None if pc[4] < 0 else (int(pc[4]), int(pc[5])))
    ro = fu.evolution_step(ops, md.TFIM(float(g["J"]), float(g["h"])), float(g["dtau"]), D,
                           fu.FullUpdate(max_iterations=8, linear_max_iterations=40), om,
                           space=None if pc[1] < 0 else (int(pc[1]), int(pc[2])), force_repair_bonds=bonds)
    assert ro["repairs"] == r["repairs"]
    assert rel(r["log_normalization_sum"], sum(v for _, v in ro["normalizations"])) < 1e-9
    en = sps.measure_energy(ps, m)
    oen = osp.measure_energy(ops, md.TFIM(float(g["J"]), float(g["h"])), om)
    assert rel(en["energy_per_site"], oen["energy_per_site"]) < 1e-9


def test_jacobi_sweep_cap_reports_nonconvergence(sps):
    """A cap of one sweep on the small-block Jacobi kernels: the SVD cannot
    confirm convergence and the call returns SPS_ERR_CONVERGENCE (5); the
    engine stays usable and gives the fixture value once the cap is lifted."""
    g = golden("pepo_2x3_D2.npz")   # 8 x 8 boundary blocks: the single-CTA Jacobi SVD
    e = _engine(sps, g)
    st = upload_golden(sps, g, e)
    m = sps.BoundaryMPS(int(g["chi0"][0]), None)
    e.set_injection(svd_sweep_cap=1)
    try:
        with pytest.raises(sps._lib.EngineError) as ei:
            sps.lognorm(st, m)
        assert ei.value.code == 5
    finally:
        e.set_injection()
    ln = sps.lognorm(st, m)
    assert rel(ln["log_norm"], g["lognorm0"][0]) < TOL


def test_born_zero_total_mass_is_an_error(sps):
    """A PEPO with a vanishing site: every conditional has zero total mass and
    the draw stops with the reference's error (born.jl:142), SPS_ERR_BORN (4),
    as the oracle does."""
    from oracle import boundary as bm, sampling as osp
    from oracle.model import State
    from oracle.z2 import T, leg
    L = 2
    sites, dims = sps.synthetic.synthetic_pepo(L, L, 2, 0.1, 3)
    sites[3] = np.zeros_like(sites[3])
    e = sps.Engine(L, L, sps.TFIM(1.0, 0.7))
    st = e.upload_state(sites, dims, True, beta=0.1)
    cache = sps.SamplingCache(st, sps.BoundaryMPS(4))
    u = np.full(L * L, 0.5)
    with pytest.raises(sps._lib.EngineError) as ei:
        sps.sample_configuration(cache, uniforms=u)
    assert ei.value.code == 4
    assert "zero total mass" in str(ei.value)
    grid = [[None] * L for _ in range(L)]
    for i, (a, d) in enumerate(zip(sites, dims)):
        grid[i % L][i // L] = T(np.asarray(a, float), [leg(int(p), int(q)) for p, q in d])
    ocache = osp.SamplingCache(State(L, L, grid, 0.1, 0.0, "pepo"), bm.BoundaryMPS(4))
    with pytest.raises(RuntimeError, match="zero total mass"):
        osp.sample_configuration(ocache, uniforms=u)
