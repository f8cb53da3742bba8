"""The physical-kind SamplingCache (the Born proposal of annealed resampling,
``src/sampling/born.jl:117-134``) on the GPU against the oracle.

A projected sample (a PEPS) is sampled over its physical labels: every
conditional weighs the two physically projected kets with the PSD-projected
site hole (``_positive_metric``, ``src/states/tensors.jl:65-94``), the last
site is bound to the PEPS's total parity, and the last row is not absorbed.
Identical configurations; log-probabilities to 1e-10 where no north boundary
is truncated, DRAW_TOL after one is (the rows after the first truncated north
absorption differ by up to 5e-8 in their conditionals on the 4x4 D=4 PEPS,
2.4e-8 relative in log p: it comes from the subspace-iteration SVD, as for
the auxiliary draws at the headline shapes; with the full-spectrum SVD they
agree to rounding, last test); the smallest relative eigenvalue of the site metrics to METRIC_TOL (the
sign of eigenvalues at the rounding level, ~1e-21 here, is solver-dependent,
so counts of clipped eigenvalues are not compared); the batched scores of
given configurations; the exhaustive distribution of a small PEPS sums to one
and vanishes on the forbidden parity.
"""
import itertools

import numpy as np
import pytest

from util import golden, upload_golden, oracle_state, rel

pytestmark = pytest.mark.gpu
TOL = 1e-10
DRAW_TOL = 1e-7
# the smallest relative eigenvalue of a site metric (about -1e-7 on the 4x4 D=4
# PEPS after a truncated north absorption): the metrics are built from the
# boundaries that carry the gap, measured 1.0e-7 apart
METRIC_TOL = 1e-6
CASES = ["pepo_2x3_D2.npz", "pepo_3x3_D4.npz", "pepo_4x4_D4.npz"]


def _projected(sps, g):
    from oracle import sampling as osp
    e = sps.Engine(int(g["Lx"]), int(g["Ly"]), sps.TFIM(float(g["J"]), float(g["h"])))
    st = upload_golden(sps, g, e)
    cfg = np.asarray(g["configs"][0])
    ps, _ = sps.project_configuration(st, cfg)
    ops, _ = osp.project_configuration(oracle_state(g), cfg.tolist())
    return e, ps, ops


def _methods(sps, g):
    from oracle import boundary as bm
    pc = g["peps_cfg"]
    chi = int(pc[3])
    space = None if pc[4] < 0 else (int(pc[4]), int(pc[5]))
    return (sps.BoundaryMPS(chi, None if space is None else sps.Z2Space(*space)), bm.BoundaryMPS(chi, space))


@pytest.mark.parametrize("case", CASES)
def test_physical_draws_match_oracle(sps, case):
    from oracle import sampling as osp
    g = golden(case)
    e, ps, ops = _projected(sps, g)
    m, om = _methods(sps, g)
    cache = sps.SamplingCache(ps, m, kind="physical")
    ocache = osp.SamplingCache(ops, om, kind="physical")
    L = int(g["Lx"]) * int(g["Ly"])
    cfgs, lps = [], []
    for seed in range(3):
        u = np.random.default_rng([11, seed]).random(L)
        d = sps.sample_configuration(cache, uniforms=u)
        od = osp.sample_configuration(ocache, uniforms=u)
        np.testing.assert_array_equal(d["configuration"], np.asarray(od["configuration"]))
        assert rel(d["log_probability"], od["log_probability"]) < DRAW_TOL
        lo = min([0.0] + [r["minimum_relative_eigenvalue"] for r in od["repairs"]
                          if "minimum_relative_eigenvalue" in r])
        assert abs(d["min_relative_eigenvalue"] - lo) < METRIC_TOL
        zero = sum(1 for r in od["repairs"] if r.get("reason") == "zero_proposal_weights")
        assert d["zero_proposals"] == zero
        cfgs.append(d["configuration"])
        lps.append(d["log_probability"])
    # the scores of given configurations, batched and concurrent, equal the draws' own
    e.set_concurrency(3)
    try:
        got, reps = sps.sample_probability_batch(cache, np.stack(cfgs))
    finally:
        e.set_concurrency(1)
    np.testing.assert_allclose(got, lps, rtol=1e-13)


def test_physical_distribution_is_normalised(sps):
    """2x3 D=2 at chi=64 (no truncation): the 64 configurations' probabilities
    sum to one; the 32 of the wrong total parity have probability zero."""
    g = golden("pepo_2x3_D2.npz")
    e, ps, ops = _projected(sps, g)
    cache = sps.SamplingCache(ps, sps.BoundaryMPS(64, None), kind="physical")
    Lx, Ly = int(g["Lx"]), int(g["Ly"])
    allc = np.array([np.array(labs).reshape(Ly, Lx).T for labs in itertools.product((1, 2), repeat=Lx * Ly)])
    lps, _ = sps.sample_probability_batch(cache, allc)
    p = np.exp(lps)
    assert np.sum(np.isneginf(lps)) == 2 ** (Lx * Ly - 1)
    assert abs(p.sum() - 1.0) < 1e-12


def test_physical_cache_needs_a_peps(sps):
    g = golden("pepo_2x3_D2.npz")
    e = sps.Engine(int(g["Lx"]), int(g["Ly"]), sps.TFIM(float(g["J"]), float(g["h"])))
    st = upload_golden(sps, g, e)
    with pytest.raises(sps._lib.EngineError):
        sps.SamplingCache(st, sps.BoundaryMPS(8), kind="physical")


@pytest.mark.parametrize("held_lambda", [None, 0.9])
def test_resampling_run_matches_the_oracle_ops(sps, monkeypatch, held_lambda):
    """run_stochastic with annealed resampling (eta_th = 1 triggers an event at
    beta = 0.3) on the device and with the oracle as the numerical ops: the
    same mixture members, fresh draws, proposal log q, selected representatives
    and curve.  held_lambda = 0.9 keeps the mixture coefficient high so that
    fresh draws come from the particles' physical-kind proposals."""
    import importlib
    import os
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from test_parallel import OracleOps
    rs = importlib.import_module(sps.__name__ + ".resample")
    if held_lambda is not None:
        real = rs.select_lambda

        def held(a, r, lam_max, tol):
            out = real(a, r, lam_max, tol)
            out["lam"] = held_lambda
            return out
        monkeypatch.setattr(rs, "select_lambda", held)
    c = sps.RunConfig(lattice=sps.Lattice(2, 2), model=sps.TFIM(1.0, 0.7), beta0=0.1, beta_log=[0.1, 0.3],
                      beta_measure=[0.1, 0.3], delta_tau_pur=0.05, delta_tau_peps=0.05, D_pur=2, D_peps=2,
                      chi_environment=4, Ns=6, seed=5,
                      resampling=sps.ResamplingOptions(enabled=True, eta_th=1.0, max_resample_sweep=2,
                                                       lambda_threshold=0.95))
    dev = sps.run_stochastic(c, sps.run_purification(c))
    ops = OracleOps(c)
    ref = sps.run_stochastic(c, sps.run_purification(c, ops=ops, identity=ops.identity), ops=ops)
    ev, oev = dev["diagnostics"]["events"][0], ref["diagnostics"]["events"][0]
    assert [s["members"] for s in ev["sweeps"]] == [s["members"] for s in oev["sweeps"]]
    for s, o in zip(ev["sweeps"], oev["sweeps"]):
        for d, od in zip(s["draws"], o["draws"]):
            np.testing.assert_array_equal(d["configuration"], od["configuration"])
            assert rel(d["log_probability"], od["log_probability"]) < 1e-9
    assert [(r["id"], r["count"]) for r in ev["post"]] == [(r["id"], r["count"]) for r in oev["post"]]
    for a, b in zip([r for r in dev["observables"]["curve"] if r.get("source") == "sampling"],
                    [r for r in ref["observables"]["curve"] if r.get("source") == "sampling"]):
        assert rel(a["lnZ"], b["lnZ"]) < 1e-9
        assert rel(a["energy_per_site"], b["energy_per_site"]) < 1e-9
        assert abs(a["eta"] - b["eta"]) < 1e-9


def test_physical_draws_with_full_spectrum_svd_match_oracle_to_rounding(sps):
    """With every truncated SVD from the full spectrum (``set_truncated_svd("full")``)
    the physical-kind draws after a truncated north absorption agree with the
    oracle to rounding (measured 9e-15 on the 4x4 D=4 PEPS): the gap of the
    default path comes from the subspace iteration."""
    from oracle import sampling as osp
    g = golden("pepo_4x4_D4.npz")
    e, ps, ops = _projected(sps, g)
    e.set_truncated_svd("full")
    m, om = _methods(sps, g)
    cache = sps.SamplingCache(ps, m, kind="physical")
    ocache = osp.SamplingCache(ops, om, kind="physical")
    for seed in range(3):
        u = np.random.default_rng([11, seed]).random(16)
        d = sps.sample_configuration(cache, uniforms=u)
        od = osp.sample_configuration(ocache, uniforms=u)
        np.testing.assert_array_equal(d["configuration"], np.asarray(od["configuration"]))
        assert rel(d["log_probability"], od["log_probability"]) < 1e-12
