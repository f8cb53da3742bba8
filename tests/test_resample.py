"""Annealed Born resampling on the host (``stopeps.jl_b200/resample.py`` and the
event in ``driver.py``), on the CPU.

The selection math against direct evaluations (mixture probabilities,
leave-one-out probabilities, the mixture coefficient against a grid search of
the same second-moment objective, SIR selection until Ns distinct members),
and one resampling run end to end with the oracle as the numerical ops
(``src/resample/event.jl``): the event's audit record, the selected
representatives and their equal weights, and reproducibility.
"""
import math
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from test_parallel import OracleOps   # noqa: E402


def _rs(sps):
    import importlib
    return importlib.import_module(sps.__name__ + ".resample")


def test_mixture_and_loo_probabilities(sps):
    rs = _rs(sps)
    assert rs.mixture_log_probability(-1.3, -0.2, 0.0) == -1.3
    v = rs.mixture_log_probability(-1.3, -0.2, 0.3)
    assert abs(v - math.log(0.7 * math.exp(-1.3) + 0.3 * math.exp(-0.2))) < 1e-14
    with pytest.raises(ValueError):
        rs.mixture_log_probability(0.0, 0.0, 1.0)
    rng = np.random.default_rng(1)
    K = 5
    mass = rng.normal(size=K)
    scores = rng.normal(size=(K, K)) - 2
    loo = rs.loo_log_probabilities(mass, scores)
    for j in range(K):
        o = [k for k in range(K) if k != j]
        ref = math.log(sum(math.exp(mass[k] + scores[k, j]) for k in o) / sum(math.exp(mass[k]) for k in o))
        assert abs(loo[j] - ref) < 1e-13


def test_select_lambda_minimises_the_second_moment(sps):
    rs = _rs(sps)
    rng = np.random.default_rng(2)
    for trial in range(5):
        a = rng.normal(size=7)
        r = rng.normal(size=7) * 2
        sel = rs.select_lambda(a, r, 0.999, 1e-8)
        off = a.max()

        def risk(lam):
            return math.log(sum(math.exp(a[j] - off) / ((1 - lam) + lam * math.exp(r[j])) for j in range(7)))
        grid = min(risk(x) for x in np.linspace(0, 0.999, 2001))
        assert 0 <= sel["lam"] <= 0.999
        assert abs(sel["log_risk_selected"] - risk(sel["lam"])) < 1e-12
        assert sel["log_risk_selected"] <= grid + 1e-7
    one = rs.select_lambda([0.3], [1.0], 0.999, 1e-8)
    assert one["lam"] == 0.0 and one["fallback"] == "single_lineage"


def test_sir_selection(sps):
    rs = _rs(sps)
    # a pool within the target keeps every member with its weight
    s = rs.sir_select_until_unique([0.0, -1.0], [1, 2], 3, seed=1, event=1)
    assert s["stop_reason"] == "pool_within_target" and s["multiplicity"] == [1, 2]
    # a larger pool: Ns distinct members, equal weights, the draw that would add another stops it
    lw = np.random.default_rng(5).normal(size=12)
    s = rs.sir_select_until_unique(lw, [1] * 12, 4, seed=3, event=2)
    assert len(s["active"]) <= 4 and sum(s["multiplicity"]) == s["Nv_post"] == len(s["selected_candidate"])
    assert all(w == 0.0 for w in s["output_relative_log_weight"])
    assert s["stop_reason"] in ("next_distinct", "draw_limit")
    assert abs(s["common_log_weight"] - (rs.logsumexp(lw) - math.log(12))) < 1e-13
    assert s == rs.sir_select_until_unique(lw, [1] * 12, 4, seed=3, event=2)


def _config(sps, **kw):
    base = dict(lattice=sps.Lattice(2, 2), model=sps.TFIM(1.0, 0.7), beta0=0.1, beta_log=[0.1, 0.3],
                beta_measure=[0.1, 0.3], delta_tau_pur=0.05, delta_tau_peps=0.05, D_pur=2, D_peps=2,
                chi_environment=4, Ns=6, seed=5,
                resampling=sps.ResamplingOptions(enabled=True, eta_th=1.0, max_resample_sweep=2))
    base.update(kw)
    return sps.RunConfig(**base)


def _run(sps, c):
    ops = OracleOps(c)
    cp = sps.run_purification(c, ops=ops, identity=ops.identity)
    return sps.run_stochastic(c, cp, ops=ops)


def test_resampling_event_end_to_end_on_the_oracle(sps):
    c = _config(sps)
    res = _run(sps, c)
    events = res["diagnostics"]["events"]
    assert events, "eta_th = 1 triggers an event"
    ev = events[0]
    assert ev["stop_reason"] in ("lambda_threshold", "sweep_limit", "no_fresh_draws")
    assert 1 <= len(ev["sweeps"]) <= 2
    for sw in ev["sweeps"]:
        assert len(sw["draws"]) == sw["M"]
        for d in sw["draws"]:
            assert math.isfinite(d["log_probability"])   # log q of the mixture proposal
    post = ev["post"]
    assert 1 <= len(post) <= c.Ns
    if ev["selection"]["stop_reason"] != "pool_within_target":
        assert all(r["relative_log_weight"] == 0.0 for r in post)
        assert sum(r["count"] for r in post) == ev["selection"]["Nv_post"]
    curve = [r for r in res["observables"]["curve"] if r.get("source") == "sampling"]
    assert all(math.isfinite(r["lnZ"]) for r in curve)
    # the same seed gives the same event
    again = _run(sps, c)["diagnostics"]["events"][0]
    assert [r["id"] for r in again["post"]] == [r["id"] for r in post]
    assert [s["members"] for s in again["sweeps"]] == [s["members"] for s in ev["sweeps"]]


def test_resampling_draws_from_member_proposals(sps, monkeypatch):
    """With the mixture coefficient held at 0.9 most fresh draws come from the
    particles' physical-kind proposals: each such draw's own probability is
    recorded as its score, and its log q mixes the baseline and member terms."""
    rs = _rs(sps)
    real = rs.select_lambda

    def held(a, r, lam_max, tol):
        out = real(a, r, lam_max, tol)
        out["lam"] = 0.9
        return out
    monkeypatch.setattr(rs, "select_lambda", held)
    c = _config(sps, resampling=sps.ResamplingOptions(enabled=True, eta_th=1.0, max_resample_sweep=1,
                                                      lambda_threshold=0.95))
    ev = _run(sps, c)["diagnostics"]["events"][0]
    sw = ev["sweeps"][0]
    assert any(m > 0 for m in sw["members"])
    entries = {(e["member_id"], e["configuration_index"]): e for e in ev["score_table"]["entries"]}
    columns = {tuple(np.asarray(x).reshape(-1).tolist()): j + 1
               for j, x in enumerate(ev["score_table"]["configurations"])}
    draws_from_members = [d for d in sw["draws"] if d["member"] > 0]
    for d in draws_from_members:
        assert math.isfinite(d["selected_log_probability"]) and math.isfinite(d["log_probability"])
        # the member's score of the drawn configuration (from the draw itself or an earlier
        # leave-one-out score of the same configuration) is the draw's own probability
        e = entries[(d["member_id"], columns[tuple(np.asarray(d["configuration"]).reshape(-1).tolist())])]
        assert abs(e["log_probability"] - d["selected_log_probability"]) < 1e-12
    for p in sw["proposals"]:
        ref = rs.mixture_log_probability(p["log_p0"], p["log_pr"], 0.9)
        assert abs(p["log_q"] - ref) < 1e-14
