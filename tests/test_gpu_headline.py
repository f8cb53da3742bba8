"""Parity at the headline shapes: D=6 (3+3), chi=36 (18+18), h=3.0, tau=0.02.

The benchmark's 8x8 lattice is too large for the CPU oracle to run in a test,
so the fixture ``headline_4x4_D6_chi36.npz`` (``tests/golden/make_golden.py``)
holds the oracle's FP64 outputs on a 4x4 lattice with the same bond, boundary
and sector dimensions (the seeded synthetic beta0 PEPO of the benchmark
workload; on 4x4 the chi=36 truncation is active in the middle bond of every
boundary after the first row).  Both absorptions are checked against their
oracle restatements: the reference's exact compression (``BoundaryMPS``) and
the zip-up variant.  Tolerances: 1e-10 relative for energies, magnetisations,
log norms and projection norms; identical Born configurations.

Two quantities carry looser, measured bounds.  Born log-probabilities agree to
1e-15 for four of the six draws; one draw per absorption differs by 1e-8
(exact compression) and 8e-6 (zip-up) relative, from the rows after the first
truncated north boundary on.  The difference comes from the subspace-iteration
SVD of the truncations (the zip-up's splits also stop at a 1e-10 residual):
with every truncated SVD from the full spectrum the exact compression's draws
agree to rounding (last test).  The bound is DRAW_TOL.  One full-update step (every ALS solve stops at its iteration limit,
so rounding is amplified by the conditioning of the reduced metrics): the
oracle's own log-normalisation moves by 7e-8 under a 1e-15 perturbation of its
input, the device differs by 3e-6; the bound is STEP_TOL.
"""
import numpy as np
import pytest

from util import golden, rel

pytestmark = pytest.mark.gpu
TOL = 1e-10
DRAW_TOL = 2e-5
STEP_TOL = 2e-5
CASE = "headline_4x4_D6_chi36.npz"


def _setup(sps):
    g = golden(CASE)
    e = sps.Engine(int(g["Lx"]), int(g["Ly"]), sps.TFIM(float(g["J"]), float(g["h"])))
    L = int(g["Lx"]) * int(g["Ly"])
    dims = g["dims"].reshape(L, 6, 2)
    sites, off = [], 0
    for i in range(L):
        n = int(np.prod([a + b for a, b in dims[i]]))
        sites.append(g["data"][off:off + n])
        off += n
    st = e.upload_state(sites, dims, True, beta=float(g["beta"]), log_amplitude=float(g["log_amplitude"]))
    return g, e, st


def _method(sps, g, tag):
    chi, a, b = (int(v) for v in g["chi"])
    kind = sps.BoundaryMPSZipUp if tag == "zip" else sps.BoundaryMPS
    return kind(chi, sps.Z2Space(a, b))


@pytest.mark.parametrize("tag", ["plain", "zip"])
def test_headline_lognorm_energy_magnetisation(sps, tag):
    g, e, st = _setup(sps)
    m = _method(sps, g, tag)
    ln = sps.lognorm(st, m)
    ref = g[f"{tag}_lognorm"]
    assert rel(ln["log_norm"], ref[0]) < TOL
    assert rel(ln["tensor_log_norm"], ref[1]) < TOL
    assert ref[2] > 0   # the chi=36 truncation is active
    assert abs(ln["max_environment_truncation"] - ref[2]) < 1e-9 * max(1.0, ref[2])
    en = sps.measure_energy(st, m, site_profile=True)
    ref = g[f"{tag}_energy"]
    assert rel(en["energy_total"], ref[0]) < TOL
    assert rel(en["energy_per_site"], ref[1]) < TOL
    assert rel(en["log_norm"], ref[2]) < TOL
    assert rel(en["x_sum"], ref[3]) < TOL
    assert rel(en["zz_sum"], ref[5]) < TOL
    np.testing.assert_allclose(en["site_x"], g[f"{tag}_site_x"], rtol=TOL, atol=TOL)
    if tag == "plain":
        # pre-truncation Schmidt entropies of the boundary compressions (BoundaryEntropy, Se profile)
        np.testing.assert_allclose(en["Se"]["north"], g["plain_Se_north"], rtol=1e-9, atol=1e-10)
        np.testing.assert_allclose(en["Se"]["south"], g["plain_Se_south"], rtol=1e-9, atol=1e-10)


@pytest.mark.parametrize("tag", ["plain", "zip"])
def test_headline_born_draws(sps, tag):
    g, e, st = _setup(sps)
    cache = sps.SamplingCache(st, _method(sps, g, tag))
    exact = 0
    for u, cfg, lp in zip(g["uniforms"], g[f"{tag}_configs"], g[f"{tag}_log_probs"]):
        d = sps.sample_configuration(cache, uniforms=u)
        np.testing.assert_array_equal(d["configuration"], cfg)
        assert rel(d["log_probability"], lp) < DRAW_TOL
        exact += rel(d["log_probability"], lp) < TOL
        d2 = sps.sample_configuration(cache, configuration=cfg)   # the probability of a given draw
        assert rel(d2["log_probability"], d["log_probability"]) < 1e-13
    assert exact >= 2
    e.set_concurrency(3)
    cfgs, lps = sps.sample_batch(cache, g["uniforms"])
    e.set_concurrency(1)
    np.testing.assert_array_equal(cfgs, g[f"{tag}_configs"])
    np.testing.assert_allclose(lps, g[f"{tag}_log_probs"], rtol=DRAW_TOL)


def test_headline_projection_and_full_update_step(sps):
    """Projection of the first draw (a D=6 PEPS) and one second-order
    full-update Trotter step of it (tau=0.02, D=6 with the (3,3) sector budget,
    exact-compression environments at chi=36), against the oracle."""
    g, e, st = _setup(sps)
    cfg = g["plain_configs"][0]
    ps, norms = sps.project_configuration(st, cfg)
    np.testing.assert_allclose(norms, g["proj_norms"], rtol=TOL, atol=TOL)
    m = _method(sps, g, "plain")
    en = sps.measure_energy(ps, m)
    assert rel(en["energy_per_site"], g["proj_energy"][0]) < TOL
    assert rel(en["log_norm"], g["proj_energy"][1]) < TOL
    D = int(g["D"])
    beta0 = ps.beta
    r = sps.evolution_step(ps, float(g["dtau"]), D, m, sps.Z2Space(D // 2, D // 2))
    assert abs(ps.beta - (beta0 + 2 * float(g["dtau"]))) < 1e-14
    assert r["bond_updates"] == int(g["step_report"][3])
    stops = [r["stop_error_tolerance"], r["stop_iteration_limit"], r["stop_residual_fallback"], r["stop_disabled"]]
    np.testing.assert_array_equal(stops, g["step_stops"])
    assert rel(r["log_normalization_sum"], float(g["step_norm_sum"])) < STEP_TOL
    assert abs(r["max_state_truncation"] - g["step_report"][0]) < STEP_TOL * max(1e-6, g["step_report"][0])
    assert abs(r["max_boundary_entropy"] - g["step_report"][2]) < STEP_TOL
    en = sps.measure_energy(ps, m, site_profile=True)
    ref = g["step_energy"]
    assert rel(en["energy_per_site"], ref[0]) < STEP_TOL
    assert rel(en["log_norm"], ref[1]) < STEP_TOL
    assert rel(en["x_sum"], ref[3]) < STEP_TOL
    np.testing.assert_allclose(en["site_x"], g["step_site_x"], rtol=STEP_TOL, atol=STEP_TOL)


def test_headline_draws_with_full_spectrum_svd(sps):
    """The exact-compression draws with every truncated SVD from the full
    spectrum: all log-probabilities to 1e-12 (measured 4e-15), where the
    default subspace iteration leaves one draw at 1e-8."""
    g, e, st = _setup(sps)
    e.set_truncated_svd("full")
    cache = sps.SamplingCache(st, _method(sps, g, "plain"))
    for u, cfg, lp in zip(g["uniforms"], g["plain_configs"], g["plain_log_probs"]):
        d = sps.sample_configuration(cache, uniforms=u)
        np.testing.assert_array_equal(d["configuration"], cfg)
        assert rel(d["log_probability"], lp) < 1e-12
