"""The CPU oracle pinned against exact diagonalization and structural invariants.

The reference ships no golden vectors (its only test checks RunConfig
validation), so exact diagonalization (``src/models/tfim.jl:72-76``,
restated in ``oracle/model.py``) and the identities below are the pins.
"""
import itertools
import math

import numpy as np
import pytest

from oracle import driver as dr, model as md, sampling as sp, boundary as bm, full_update as fu
from util import golden


def _cfg(**kw):
    base = dict(Lx=2, Ly=2, J=1.0, h=0.7, beta0=0.2, beta_log=[0.1, 0.2], beta_measure=[0.0, 0.2],
                delta_tau_pur=0.025, delta_tau_peps=0.025, D_pur=4, D_peps=4, chi_environment=16, Ns=4, seed=1)
    base.update(kw)
    return dr.RunConfig(**base)


def test_identity_pepo_norm_is_hilbert_dimension():
    st = md.identity_pepo(3, 2)
    md.normalize_state(st)
    ln = bm.lognorm(st, bm.BoundaryMPS(4))
    assert abs(ln["log_norm"] - 6 * math.log(2)) < 1e-13
    assert abs(sp.measure_energy(st, md.TFIM(1.0, 0.7), bm.BoundaryMPS(4))["energy_per_site"]) < 1e-14


@pytest.mark.parametrize("h", [0.7, 3.0])
def test_purification_matches_exact_diagonalization(h):
    c = _cfg(h=h)
    st, rows = dr.run_purification(c)
    for r in rows:
        ex = md.exact_thermal_observables(2, 2, md.TFIM(1.0, h), r["beta"])
        tol = 2e-5 * max(1.0, h * h)   # second-order Trotter error at delta_tau = 0.025
        assert abs(r["lnZ"] - ex["lnZ"]) < tol
        if not math.isnan(r["energy_per_site"]):
            assert abs(r["energy_per_site"] - ex["energy_per_site"]) < tol
            mx = md.exact_thermal_magnetization(2, 2, md.TFIM(1.0, h), r["beta"])
            assert abs(r["magnetization"] - mx) < tol


def test_purification_3x3_converges_to_exact_diagonalization():
    """3x3 at h=3.0 (512-state exact diagonalization, restating tfim.jl:72-76):
    lnZ, energy and magnetisation per site after purification to beta=0.2 at
    D=4, chi=16 agree with ED within the second-order Trotter error, and
    halving delta_tau cuts the error by about four (measured 4.2, 4.6, 4.2), so
    the boundary truncations and the full update add nothing visible."""
    errs = {}
    for tau in (0.025, 0.0125):
        c = _cfg(Lx=3, Ly=3, h=3.0, delta_tau_pur=tau, delta_tau_peps=tau, beta_measure=[0.1, 0.2])
        st, rows = dr.run_purification(c)
        r = rows[-1]
        assert abs(r["beta"] - 0.2) < 1e-12
        ex = md.exact_thermal_observables(3, 3, md.TFIM(1.0, 3.0), 0.2)
        mx = md.exact_thermal_magnetization(3, 3, md.TFIM(1.0, 3.0), 0.2)
        errs[tau] = (abs(r["lnZ"] - ex["lnZ"]) / 9, abs(r["energy_per_site"] - ex["energy_per_site"]),
                     abs(r["magnetization"] - mx))
    for e in errs[0.025]:
        assert e < 1e-4
    for coarse, fine in zip(errs[0.025], errs[0.0125]):
        assert 3.0 < coarse / fine < 6.0


def _site_x_exact(Lx, Ly, m, beta):
    """<X_i> per site at inverse temperature beta by exact diagonalization."""
    H = md.dense_hamiltonian(Lx, Ly, m)
    e, V = np.linalg.eigh(H)
    w = np.exp(-beta * (e - e.min()))
    b = np.arange(1 << (Lx * Ly))
    out = []
    for i in range(Lx * Ly):
        Xi = np.zeros_like(H)
        Xi[b ^ (1 << i), b] = 1.0
        out.append(float(w @ np.einsum("ik,ij,jk->k", V, Xi, V) / w.sum()))
    return np.array(out)


def test_per_site_fields_converge_to_exact_diagonalization():
    """The per-site-field TFIM (an extension for per-site gradients; the
    reference has one h): purification to beta=0.2 converges to the per-site ED
    at second order in delta_tau, and the central difference of lnZ in h_i
    (step 1e-4) gives beta <X_i> (the exact derivative) within the Trotter error."""
    rng = np.random.default_rng(7)
    fields = tuple(3.0 + rng.uniform(-0.5, 0.5, 6))
    errs = []
    for tau in (0.025, 0.0125):
        c = _cfg(Lx=3, Ly=2, h=3.0, fields=fields, delta_tau_pur=tau, delta_tau_peps=tau)
        r = dr.run_purification(c)[1][-1]
        ex = md.exact_thermal_observables(3, 2, md.TFIM(1.0, 3.0, fields), 0.2)
        errs.append(abs(r["energy_per_site"] - ex["energy_per_site"]))
    assert errs[0] < 1e-4 and 3.0 < errs[0] / errs[1] < 6.0
    f2 = tuple(3.0 + rng.uniform(-0.5, 0.5, 4))
    exact = 0.2 * _site_x_exact(2, 2, md.TFIM(1.0, 3.0, f2), 0.2)
    step = 1e-4
    for i in range(4):
        lz = []
        for s in (+1, -1):
            f = list(f2)
            f[i] += s * step
            lz.append(dr.run_purification(_cfg(h=3.0, fields=tuple(f), delta_tau_pur=0.0125))[1][-1]["lnZ"])
        assert abs((lz[0] - lz[1]) / (2 * step) - exact[i]) < 1e-5   # measured 2.4e-6 (4.8e-7 at tau/2)


def test_born_probabilities_sum_to_one_and_weights_give_Z():
    """Exhaustive 2x2: sum_k p_k = 1 and sum_k ||psi_k||^2 = Z(beta0) = ||PEPO||^2."""
    c = _cfg()
    st, rows = dr.run_purification(c)
    cache = sp.SamplingCache(st, bm.BoundaryMPS(16))
    total_p, total_w = 0.0, 0.0
    for bits in itertools.product([1, 2], repeat=4):
        cfg = [[bits[0], bits[2]], [bits[1], bits[3]]]
        d = sp.sample_configuration(cache, configuration=cfg)
        total_p += math.exp(d["log_probability"])
        ps, _ = sp.project_configuration(st, cfg)
        total_w += math.exp(bm.lognorm(ps, bm.BoundaryMPS(16))["log_norm"])
    assert abs(total_p - 1.0) < 1e-12
    assert abs(math.log(total_w) - rows[-1]["lnZ"]) < 1e-12


def test_exhaustive_ensemble_reproduces_exact_energy():
    """Weighting every configuration by its evolved norm reproduces the ED energy at beta."""
    c = _cfg(beta0=0.1, beta_log=[0.1], beta_measure=[0.1])
    st, _ = dr.run_purification(c)
    beta = 0.3
    num = den = 0.0
    for bits in itertools.product([1, 2], repeat=4):
        cfg = [[bits[0], bits[2]], [bits[1], bits[3]]]
        ps, _ = sp.project_configuration(st, cfg)
        rep = dr.evolve(ps, c, dr.step_schedule(0.1, beta, 0.025), 4, None)
        m = sp.measure_energy(ps, md.TFIM(1.0, 0.7), bm.BoundaryMPS(16))
        w = math.exp(m["log_norm"])
        num += w * m["energy_per_site"]
        den += w
    ex = md.exact_thermal_observables(2, 2, md.TFIM(1.0, 0.7), beta)
    assert abs(num / den - ex["energy_per_site"]) < 5e-5


def test_stochastic_estimate_is_consistent_with_exact():
    c = _cfg(Ns=24, beta_log=[0.2, 0.4], beta_measure=[0.2, 0.4], delta_tau_pur=0.05, delta_tau_peps=0.05)
    st, _ = dr.run_purification(c)
    res = dr.run_stochastic(c, st)
    for r in res["curve"]:
        ex = md.exact_thermal_observables(2, 2, md.TFIM(1.0, 0.7), r["beta"])
        assert abs(r["energy_per_site"] - ex["energy_per_site"]) < 4 * r["energy_per_site_error"] + 1e-3


def test_categorical_matches_reference_rule():
    lm = [math.log(0.25), math.log(0.75)]
    assert sp.categorical(lm, 0.2) == 0
    assert sp.categorical(lm, 0.3) == 1
    assert sp.categorical([-math.inf, 0.0], 0.99) == 1


def test_truncation_is_an_intersection():
    from oracle.z2 import select_truncation
    s = [np.array([10.0, 9, 8, 7]), np.array([1.0, 0.5])]
    keep = select_truncation(s, chi=5, space=(3, 3))
    assert keep[0].tolist() == [True, True, True, False] and keep[1].tolist() == [True, False]


@pytest.mark.parametrize("name", ["pepo_3x3_D4.npz", "pepo_2x3_D2.npz"])
def test_golden_fixture_is_reproducible(name):
    """The committed fixtures are what the oracle computes today."""
    from util import oracle_state, space
    g = golden(name)
    st = oracle_state(g)
    for k in range(2):
        a, b, cc = g[f"chi{k}"]
        m = bm.BoundaryMPS(int(a), space(b, cc))
        ln = bm.lognorm(st, m)
        assert abs(ln["log_norm"] - g[f"lognorm{k}"][0]) < 1e-11
    a, b, cc = g["chi0"]
    cache = sp.SamplingCache(st, bm.BoundaryMPS(int(a), space(b, cc)))
    d = sp.sample_configuration(cache, uniforms=g["uniforms"][0])
    assert np.array_equal(np.asarray(d["configuration"]), g["configs"][0])


@pytest.mark.parametrize("name", ["pepo_2x3_D2.npz"])
def test_zipup_equals_exact_compression_without_truncation(name):
    """With chi above the exact boundary bond (d = D^2 = 4 for a 2-wide D=2 lattice) neither absorption
    truncates, so the zip-up restatement must give the plain compression's norm and the same Born draws."""
    from util import oracle_state
    g = golden(name)
    st = oracle_state(g)
    plain, zip_ = bm.BoundaryMPS(16), bm.BoundaryMPS(16, None, zipup=True)
    a, b = bm.lognorm(st, plain), bm.lognorm(st, zip_)
    assert abs(a["log_norm"] - b["log_norm"]) < 1e-12 * max(1.0, abs(a["log_norm"]))
    cp, cz = sp.SamplingCache(st, plain), sp.SamplingCache(st, zip_)
    for u in g["uniforms"][:2]:
        dp = sp.sample_configuration(cp, uniforms=u)
        dz = sp.sample_configuration(cz, uniforms=u)
        assert np.array_equal(np.asarray(dp["configuration"]), np.asarray(dz["configuration"]))
        assert abs(dp["log_probability"] - dz["log_probability"]) < 1e-11 * max(1.0, abs(dp["log_probability"]))


def test_physical_proposal_is_the_born_distribution_of_the_peps():
    """The physical-kind proposal (``born.jl:117-134``) on a projected 2x3 D=2
    PEPS contracted exactly (chi=64): every configuration's probability is
    |psi(s)|^2 / <psi|psi> (the PEPS with its physical legs fixed, contracted
    on its own), the parity-forbidden half has probability zero, and the
    probabilities sum to one."""
    from oracle.model import State
    from util import oracle_state
    g = golden("pepo_2x3_D2.npz")
    ps, _ = sp.project_configuration(oracle_state(g), np.asarray(g["configs"][0]).tolist())
    m = bm.BoundaryMPS(64, None)
    cache = sp.SamplingCache(ps, m, kind="physical")
    ln0 = bm.lognorm(ps, m)["tensor_log_norm"]
    Lx, Ly = ps.Lx, ps.Ly
    total, nonzero = 0.0, 0
    for labs in itertools.product((1, 2), repeat=Lx * Ly):
        conf = [[labs[x + y * Lx] for y in range(Ly)] for x in range(Lx)]
        lp = sp.sample_configuration(cache, configuration=conf)["log_probability"]
        if lp == -math.inf:
            continue
        nonzero += 1
        total += math.exp(lp)
        sites = [[sp.project_physical(ps[x, y], conf[x][y] - 1) for y in range(Ly)] for x in range(Lx)]
        exact = bm.lognorm(State(Lx, Ly, sites, ps.beta, 0.0, "peps"), m)["tensor_log_norm"] - ln0
        assert abs(math.exp(lp) - math.exp(exact)) <= 1e-12 * math.exp(exact)
    assert nonzero == 2 ** (Lx * Ly - 1)
    assert abs(total - 1.0) < 1e-12
    # a draw from uniforms has the probability of its configuration
    d = sp.sample_configuration(cache, uniforms=np.random.default_rng(3).random(Lx * Ly))
    again = sp.sample_configuration(cache, configuration=d["configuration"])
    assert abs(d["log_probability"] - again["log_probability"]) < 1e-13
    assert len([r for r in d["repairs"] if "minimum_relative_eigenvalue" in r]) == Lx * Ly
