"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Every value is compared with the oracle's FP64 output on the same inputs:
golden fixtures from ``tests/golden/make_golden.py`` and, for the larger
checks, the oracle run live.  Tolerance: 1e-10 relative (the plain-path bar);
Born draws must select identical configurations from identical uniforms.
"""
import math

import numpy as np
import pytest

from util import golden, upload_golden, oracle_state, space, rel

pytestmark = pytest.mark.gpu
TOL = 1e-10
# Born log-probabilities of the zip-up absorption: its truncated SVDs stop at a
# 1e-10 relative residual (the splits' stopping rule), which moves a draw's
# log p by up to a few 1e-10 on the purified 4x4 D=4 PEPO, whose boundary
# spectra decay fast (measured 3.0e-10 for one of its draws)
ZIP_LOGP_TOL = 1e-9

CASES = ["pepo_3x3_D4.npz", "pepo_2x3_D2.npz", "pepo_4x4_D4.npz"]


def _engine(sps, g, **kw):
    return sps.Engine(int(g["Lx"]), int(g["Ly"]), sps.TFIM(float(g["J"]), float(g["h"])), **kw)


def _bmps(sps, a, b, c):
    return sps.BoundaryMPS(int(a), None if b < 0 else sps.Z2Space(int(b), int(c)))


@pytest.mark.parametrize("case", CASES)
def test_lognorm_and_energy(sps, case):
    g = golden(case)
    e = _engine(sps, g)
    st = upload_golden(sps, g, e)
    for k in range(2):
        m = _bmps(sps, *g[f"chi{k}"])
        ln = sps.lognorm(st, m)
        ref = g[f"lognorm{k}"]
        assert rel(ln["log_norm"], ref[0]) < TOL
        assert rel(ln["tensor_log_norm"], ref[1]) < TOL
        assert abs(ln["max_environment_truncation"] - ref[2]) < 1e-9
        en = sps.measure_energy(st, m, site_profile=True)
        ref = g[f"energy{k}"]
        assert rel(en["energy_total"], ref[0]) < TOL
        assert rel(en["energy_per_site"], ref[1]) < TOL
        assert rel(en["log_norm"], ref[2]) < TOL
        assert rel(en["x_sum"], ref[3]) < TOL
        np.testing.assert_allclose(en["site_x"], g[f"site_x{k}"], rtol=TOL, atol=TOL)


@pytest.mark.parametrize("case", CASES)
def test_born_draws(sps, case):
    g = golden(case)
    e = _engine(sps, g)
    st = upload_golden(sps, g, e)
    cache = sps.SamplingCache(st, _bmps(sps, *g["chi0"]))
    for u, cfg, lp in zip(g["uniforms"], g["configs"], g["log_probs"]):
        d = sps.sample_configuration(cache, uniforms=u)
        np.testing.assert_array_equal(d["configuration"], cfg)
        assert rel(d["log_probability"], lp) < TOL
        # configuration= evaluates the same probability (born.jl:89-93,145)
        d2 = sps.sample_configuration(cache, configuration=cfg)
        assert rel(d2["log_probability"], lp) < TOL
    cfgs, lps = sps.sample_batch(cache, g["uniforms"])
    np.testing.assert_array_equal(cfgs, g["configs"])
    np.testing.assert_allclose(lps, g["log_probs"], rtol=TOL)


@pytest.mark.parametrize("case", CASES)
def test_projection(sps, case):
    """project_configuration (born.jl:27-36): the per-site normalisations and
    the projected PEPS's energy and log norm; the step itself is
    test_evolution_step."""
    g = golden(case)
    e = _engine(sps, g)
    st = upload_golden(sps, g, e)
    pc = g["peps_cfg"]
    ps, norms = sps.project_configuration(st, g["configs"][0])
    np.testing.assert_allclose(norms, g["proj_norms"], rtol=TOL, atol=TOL)
    m = _bmps(sps, pc[3], pc[4], pc[5])
    en = sps.measure_energy(ps, m)
    assert rel(en["energy_per_site"], g["proj_energy"][0]) < TOL
    assert rel(en["log_norm"], g["proj_energy"][1]) < TOL
    assert not ps.is_pepo


@pytest.mark.parametrize("case", CASES)
def test_evolution_step(sps, case):
    """One second-order full-update step of a projected PEPS against the
    oracle's fixture: bond count, stop reasons, the log normalisation and the
    stepped state's energy, log norm and <X> at 1e-9.  The bar is looser than
    the contraction's 1e-10 because each ALS solve is an iterative Jacobi-PCG
    (full_update.jl:371-400) that stops at a relative residual of 1e-9 (the
    FullUpdate linear tolerance): device and oracle take the same iterations,
    but their rounding moves the stopping residual at that level."""
    g = golden(case)
    upd = sps.FullUpdate(max_iterations=8, linear_max_iterations=40) if "2x3" in case else sps.FullUpdate()
    e = _engine(sps, g, update=upd)
    st = upload_golden(sps, g, e)
    pc = g["peps_cfg"]
    ps, _ = sps.project_configuration(st, g["configs"][0])
    m = _bmps(sps, pc[3], pc[4], pc[5])
    sp = None if pc[1] < 0 else sps.Z2Space(int(pc[1]), int(pc[2]))
    beta0 = ps.beta
    r = sps.evolution_step(ps, float(g["dtau"]), int(pc[0]), m, sp)
    assert r["bond_updates"] == int(g["step_report"][3])
    assert abs(ps.beta - (beta0 + 2 * float(g["dtau"]))) < 1e-14
    stops = [r["stop_error_tolerance"], r["stop_iteration_limit"], r["stop_residual_fallback"], r["stop_disabled"]]
    np.testing.assert_array_equal(stops, g["step_stops"])
    assert rel(r["log_normalization_sum"], float(g["step_norm_sum"])) < 1e-9
    en = sps.measure_energy(ps, m)
    ref = g["step_energy"]
    assert rel(en["energy_per_site"], ref[0]) < 1e-9
    assert rel(en["log_norm"], ref[1]) < 1e-9
    assert rel(en["x_sum"], ref[3]) < 1e-9


def test_pipeline_2x2(sps):
    g = golden("pipeline_2x2.npz")
    c = sps.RunConfig(lattice=sps.Lattice(2, 2), model=sps.TFIM(1.0, 0.7), beta0=0.2, beta_log=[0.1, 0.2, 0.3],
                      beta_measure=[0.2, 0.3], delta_tau_pur=0.05, delta_tau_peps=0.05, D_pur=2, D_peps=2,
                      bond_space_pur=sps.Z2Space(1, 1), bond_space_peps=sps.Z2Space(1, 1), chi_environment=4,
                      environment_space=sps.Z2Space(2, 2), Ns=6, seed=3,
                      resampling=sps.ResamplingOptions(enabled=False))
    cp = sps.run_purification(c)
    np.testing.assert_allclose([r["lnZ"] for r in cp.purification], g["pur_lnZ"], rtol=1e-9)
    res = sps.run_stochastic(c, cp)
    draws = res["diagnostics"]["born_draws"]
    np.testing.assert_array_equal(np.stack([d["configuration"] for d in draws]), g["draw_cfg"])
    np.testing.assert_allclose([d["log_probability"] for d in draws], g["draw_logp"], rtol=1e-9)
    curve = [r for r in res["observables"]["curve"] if r.get("source") == "sampling"]
    np.testing.assert_allclose([r["energy_per_site"] for r in curve], g["energy"], rtol=1e-9)
    np.testing.assert_allclose([r["lnZ"] for r in curve], g["lnZ"], rtol=1e-9)
    np.testing.assert_allclose([r["eta"] for r in curve], g["eta"], rtol=1e-9)
    assert res["metadata"]["complete"]


def test_live_oracle_3x3_chi_truncating(sps):
    """A fresh purification on device and oracle with truncating boundaries (chi=6)."""
    from oracle import driver as odr
    kw = dict(beta0=0.1, beta_log=[0.1], beta_measure=[0.1], delta_tau_pur=0.05, D_pur=3, D_peps=3,
              chi_environment=6, Ns=1)
    c = sps.RunConfig(lattice=sps.Lattice(3, 3), model=sps.TFIM(1.0, 1.3), **kw,
                      resampling=sps.ResamplingOptions(enabled=False))
    oc = odr.RunConfig(Lx=3, Ly=3, J=1.0, h=1.3, **kw)
    cp = sps.run_purification(c)
    _, rows = odr.run_purification(oc)
    assert rel(cp.purification[-1]["lnZ"], rows[-1]["lnZ"]) < 1e-9
    assert rel(cp.purification[-1]["energy_per_site"], rows[-1]["energy_per_site"]) < 1e-9
    assert rel(cp.purification[-1]["magnetization"], rows[-1]["magnetization"]) < 1e-9


def test_error_status_is_raised(sps):
    e = sps.Engine(2, 2)
    st = e.identity_pepo()
    with pytest.raises(ValueError):
        sps.sample_configuration(sps.SamplingCache(st, sps.BoundaryMPS(4)))
    with pytest.raises(sps._lib.EngineError):
        sps.lognorm(st, sps.BoundaryMPS(0))


@pytest.mark.parametrize("case", CASES)
def test_zipup_draws_and_energy(sps, case):
    """The zip-up absorption against its oracle restatement (energy and log
    norm to 1e-10, log p to ZIP_LOGP_TOL), and against the reference's exact compression within
    the precision target of the batched path (energy per site within 1e-4)."""
    from oracle import boundary as bm, model as md, sampling as osp
    g = golden(case)
    e = _engine(sps, g)
    st = upload_golden(sps, g, e)
    chi, a, b = (int(v) for v in g["chi0"])
    osp_space = None if a < 0 else (a, b)
    zm = sps.BoundaryMPSZipUp(chi, None if a < 0 else sps.Z2Space(a, b))
    ost = oracle_state(g)
    ocache = osp.SamplingCache(ost, bm.BoundaryMPS(chi, osp_space, zipup=True))
    cache = sps.SamplingCache(st, zm)
    for u, cfg in zip(g["uniforms"], g["configs"]):
        d = sps.sample_configuration(cache, uniforms=u)
        od = osp.sample_configuration(ocache, uniforms=u)
        np.testing.assert_array_equal(d["configuration"], np.asarray(od["configuration"]))
        assert rel(d["log_probability"], od["log_probability"]) < ZIP_LOGP_TOL
    model = md.TFIM(float(g["J"]), float(g["h"]))
    oe = osp.measure_energy(ost, model, bm.BoundaryMPS(chi, osp_space, zipup=True))
    en = sps.measure_energy(st, zm)
    assert rel(en["energy_per_site"], oe["energy_per_site"]) < TOL
    assert rel(en["log_norm"], oe["log_norm"]) < TOL
    assert abs(en["energy_per_site"] - g["energy0"][1]) < 1e-4


@pytest.mark.parametrize("case", ["pepo_4x4_D4.npz"])
def test_concurrent_batch_matches_serial(sps, case):
    """Samples drawn concurrently (own stream and workspace each, shared cache)
    are the serial draws: same configurations, log-probabilities to rounding."""
    g = golden(case)
    e = _engine(sps, g)
    st = upload_golden(sps, g, e)
    for m in (_bmps(sps, *g["chi0"]),
              sps.BoundaryMPSZipUp(int(g["chi0"][0]), _bmps(sps, *g["chi0"]).sector_space)):
        cache = sps.SamplingCache(st, m)
        u = np.stack([sps.sample_uniforms(3, i, int(g["Lx"]) * int(g["Ly"])) for i in range(1, 8)])
        e.set_concurrency(1)
        c1, l1 = sps.sample_batch(cache, u)
        e.set_concurrency(3)
        c3, l3 = sps.sample_batch(cache, u)
        e.set_concurrency(1)
        np.testing.assert_array_equal(c1, c3)
        np.testing.assert_allclose(l1, l3, rtol=1e-12)


def test_rank_deficient_boundary(sps):
    """A PEPO whose boundary blocks have rank 1 (the identity thermal factor in
    D = 4 bonds): the subspace-iteration SVD deflates the columns at the
    rounding level and completes the vectors of the zero values (or, for
    blocks too small for it, the full Jacobi SVD runs); both absorptions agree
    with the oracle."""
    from oracle import boundary as bm
    from oracle.model import State
    from oracle.z2 import T, leg
    L = 4
    sites, dims = sps.synthetic.synthetic_pepo(L, L, 4, 0.0, 7)
    e = sps.Engine(L, L, sps.TFIM(1.0, 0.7))
    st = e.upload_state(sites, dims, True, beta=0.0)
    grid = [[None] * L for _ in range(L)]
    for i, (a, d) in enumerate(zip(sites, dims)):
        grid[i % L][i // L] = T(np.asarray(a, float), [leg(int(p), int(q)) for p, q in d])
    ost = State(L, L, grid, 0.0, 0.0, "pepo")
    for zip_up in (False, True):
        kind = sps.BoundaryMPSZipUp if zip_up else sps.BoundaryMPS
        ln = sps.lognorm(st, kind(16, sps.Z2Space(8, 8)))
        ref = bm.lognorm(ost, bm.BoundaryMPS(16, (8, 8), zipup=zip_up))
        # the normalised product state: log norm 0 (absolute comparison)
        assert abs(ln["log_norm"] - ref["log_norm"]) < 1e-10
        assert abs(ln["tensor_log_norm"] - ref["tensor_log_norm"]) < 1e-10


@pytest.mark.parametrize("zip_up", [False, True])
def test_truncrank_without_sector_budget(sps, zip_up):
    """truncrank(chi) with sector_space = nothing: the kept values are chosen
    across both parity blocks (the subspace-iteration SVD computes chi per
    block), against the oracle run live on the 4x4 D=4 fixture."""
    from oracle import boundary as bm, model as md, sampling as osp
    g = golden("pepo_4x4_D4.npz")
    e = _engine(sps, g)
    st = upload_golden(sps, g, e)
    ost = oracle_state(g)
    kind = sps.BoundaryMPSZipUp if zip_up else sps.BoundaryMPS
    ln = sps.lognorm(st, kind(16, None))
    ref = bm.lognorm(ost, bm.BoundaryMPS(16, None, zipup=zip_up))
    assert rel(ln["log_norm"], ref["log_norm"]) < TOL
    assert abs(ln["max_environment_truncation"] - ref["max_environment_truncation"]) < 1e-9
    en = sps.measure_energy(st, kind(16, None))
    oen = osp.measure_energy(ost, md.TFIM(float(g["J"]), float(g["h"])), bm.BoundaryMPS(16, None, zipup=zip_up))
    assert rel(en["energy_per_site"], oen["energy_per_site"]) < TOL


def test_config1_end_to_end(sps):
    """The plain-method configuration (4x4 TFIM h=0.7, D=4 = 2+2, chi=16 = 8+8,
    tau=0.05, beta0=0.5, seed 1) end to end: purification, four Born draws,
    full-update evolution of the unique configurations to beta=1 and the
    ensemble curve, against the oracle's run (fixture config1_4x4_D4_run.npz)."""
    import os
    from util import GOLDEN
    if not os.path.exists(os.path.join(GOLDEN, "config1_4x4_D4_run.npz")):
        pytest.skip("fixture not generated")
    g = golden("config1_4x4_D4_run.npz")
    c = sps.RunConfig(lattice=sps.Lattice(4, 4), model=sps.TFIM(1.0, 0.7), beta0=0.5, beta_log=[1.0],
                      beta_measure=[0.5, 1.0], delta_tau_pur=0.05, delta_tau_peps=0.05, D_pur=4, D_peps=4,
                      bond_space_pur=sps.Z2Space(2, 2), bond_space_peps=sps.Z2Space(2, 2), chi_environment=16,
                      environment_space=sps.Z2Space(8, 8), Ns=4, seed=1,
                      resampling=sps.ResamplingOptions(enabled=False))
    cp = sps.run_purification(c)
    np.testing.assert_allclose([r["lnZ"] for r in cp.purification], g["pur_lnZ"], rtol=1e-9)
    res = sps.run_stochastic(c, cp)
    draws = res["diagnostics"]["born_draws"]
    np.testing.assert_array_equal(np.stack([d["configuration"] for d in draws]), g["draw_cfg"])
    np.testing.assert_allclose([d["log_probability"] for d in draws], g["draw_logp"], rtol=1e-9)
    curve = [r for r in res["observables"]["curve"] if r.get("source") == "sampling"]
    np.testing.assert_allclose([r["beta"] for r in curve], g["beta"], rtol=1e-14)
    np.testing.assert_allclose([r["energy_per_site"] for r in curve], g["energy"], rtol=1e-8)
    np.testing.assert_allclose([r["lnZ"] for r in curve], g["lnZ"], rtol=1e-8)
    np.testing.assert_allclose([r["eta"] for r in curve], g["eta"], rtol=1e-8)
