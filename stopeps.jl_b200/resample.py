"""Annealed Born resampling: the host side of one resampling event.

Restates ``src/resample/selection.jl`` (mixture probabilities, leave-one-out
proposal probabilities, the choice of the mixture coefficient, sampling
importance resampling until Ns distinct representatives),
``src/resample/scores.jl`` (the table of configuration probabilities of an
event) and ``src/resample/event.jl`` (the resampling plan, fresh draws from
the mixture proposal, their replay through the evolution history, the pool
selection).  The numerical work -- physical-kind SamplingCaches of the
particles' PEPS, draws, configuration probabilities, projections, evolution
and measurement -- goes through the drivers' ops (the device engine by
default).  The reference's ``_event_rng(seed, domain, event, item)`` streams
are replaced by explicit uniforms from ``event_uniforms`` (numpy's
default_rng on the same four integers), as ``sample_uniforms`` replaces
``sample_rng``.
"""
from __future__ import annotations

import math

import numpy as np

# stream domains of event_uniforms (the reference's _event_rng domain words)
DOMAIN_SIR_SLOT = 1      # SIR selection draws (selection.jl:84)
DOMAIN_MIXTURE = 2       # choice of the mixture component of a fresh draw (event.jl:117)
DOMAIN_FRESH = 3         # the Born draw of a fresh sample (event.jl:126)


def event_uniforms(seed: int, domain: int, event: int, item: int, n: int) -> np.ndarray:
    """n uniforms of the stream (seed, domain, event, item)."""
    if seed < 0 or event < 1 or item < 1:
        raise ValueError("invalid random stream identity")
    return np.random.default_rng([int(seed), int(domain), int(event), int(item)]).random(n)


def logsumexp(x) -> float:
    """``_rs_logsumexp`` (``selection.jl:1-7``)."""
    x = list(x)
    if not x:
        return -math.inf
    pivot = max(x)
    if pivot == -math.inf:
        return -math.inf
    if not math.isfinite(pivot):
        raise ValueError("nonfinite positive log mass")
    return pivot + math.log(sum(math.exp(v - pivot) for v in x))


def mixture_log_probability(log_p0: float, log_pr, lam: float) -> float:
    """``_mixture_log_probability`` (``selection.jl:9-14``): log((1-lam) p0 + lam pr)."""
    if not 0 <= lam < 1:
        raise ValueError("invalid resampling mixture coefficient")
    if lam == 0:
        return float(log_p0)
    return logsumexp([math.log1p(-lam) + log_p0, math.log(lam) + log_pr])


def loo_log_probabilities(log_mass, scores):
    """``_loo_log_probabilities`` (``selection.jl:17-26``): for each member j the
    log-probability of its configuration under the mixture of the other
    members' proposals, weighted by their masses (scores[k, j] = log p_k(x_j))."""
    log_mass = np.asarray(log_mass, float)
    scores = np.asarray(scores, float)
    K = len(log_mass)
    if scores.shape != (K, K):
        raise ValueError("LOO scores must be K by K")
    out = []
    for j in range(K):
        others = [k for k in range(K) if k != j]
        num = logsumexp([log_mass[k] + scores[k, j] for k in others])
        out.append(num - (logsumexp([log_mass[k] for k in others]) if others else 0.0))
    return np.asarray(out)


def select_lambda(log_amplitude_squared, log_ratio, lambda_max: float, lambda_tolerance: float):
    """``_select_lambda`` (``selection.jl:29-66``): the mixture coefficient in
    [0, lambda_max] minimising the estimated second moment
    sum_j a_j / ((1 - lam) + lam r_j), by golden-section search; the midpoint
    of the last bracket competes with both ends, the smaller coefficient wins
    ties within 64 eps."""
    a = np.asarray(log_amplitude_squared, float)
    r = np.asarray(log_ratio, float)
    if not (len(a) == len(r) > 0):
        raise ValueError("invalid LOO arrays")
    if not (np.all(np.isfinite(a)) and all(math.isfinite(v) or v == -math.inf for v in r)):
        raise ValueError("invalid LOO risk or probability ratio")
    offset = float(a.max())
    amp = a - offset

    def risk(lam):
        return logsumexp([amp[j] - mixture_log_probability(0.0, r[j], lam) for j in range(len(amp))])

    if len(amp) == 1 or lambda_max == 0:
        return dict(lam=0.0, log_risk_offset=offset, log_risk_zero=risk(0.0), log_risk_selected=risk(0.0),
                    log_risk_upper=risk(lambda_max), fallback="single_lineage" if len(amp) == 1 else "zero_interval")
    left, right = 0.0, lambda_max
    golden = (math.sqrt(5.0) - 1) / 2
    x1, x2 = right - golden * (right - left), left + golden * (right - left)
    f1, f2 = risk(x1), risk(x2)
    while right - left > lambda_tolerance:
        if f1 <= f2:
            right, x2, f2 = x2, x1, f1
            x1 = right - golden * (right - left)
            f1 = risk(x1)
        else:
            left, x1, f1 = x1, x2, f2
            x2 = left + golden * (right - left)
            f2 = risk(x2)
    candidates = sorted([0.0, (left + right) / 2, lambda_max])
    risks = [risk(x) for x in candidates]
    best = min(risks)
    tie = 64 * float(np.spacing(max(1.0, max(abs(v) for v in risks))))
    index = next(i for i, v in enumerate(risks) if v <= best + tie)
    return dict(lam=candidates[index], log_risk_offset=offset, log_risk_zero=risks[0],
                log_risk_selected=risks[index], log_risk_upper=risks[-1], fallback="none")


def categorical(log_mass, u: float) -> int:
    """``_categorical`` (``selection.jl:68-80``) with the uniform supplied (0-based)."""
    z = logsumexp(log_mass)
    if not math.isfinite(z):
        raise ValueError("proposal requires positive total probability")
    cumulative, last = 0.0, -1
    for j, v in enumerate(log_mass):
        if v == -math.inf:
            continue
        last = j
        cumulative += math.exp(v - z)
        if u < cumulative:
            return j
    return last


def sir_select_until_unique(log_weight, multiplicity, Ns: int, seed: int, event: int):
    """``_sir_select_until_unique`` (``selection.jl:83-120``): draw pool members
    with probability proportional to weight x multiplicity, one uniform per
    slot (stream DOMAIN_SIR_SLOT), until Ns distinct members are held and the
    next draw would add another (or 3 Ns draws); the selected members carry
    equal weights.  A pool of at most Ns members is kept as it is."""
    lw = np.asarray(log_weight, float)
    mult = [int(m) for m in multiplicity]
    if not (isinstance(Ns, (int, np.integer)) and Ns >= 1):
        raise ValueError("invalid representative target")
    if not (len(lw) == len(mult) > 0):
        raise ValueError("empty or inconsistent SIR pool")
    if not np.all(np.isfinite(lw)):
        raise ValueError("pool weights must be finite")
    if not all(m > 0 for m in mult):
        raise ValueError("pool multiplicities must be positive integers")
    K, Nv = len(lw), sum(mult)
    if K <= Ns:
        return dict(selected_candidate=[], multiplicity=list(mult), active=list(range(K)), common_log_weight=0.0,
                    output_relative_log_weight=lw.tolist(), draw_count=0, discarded_candidate=None,
                    stop_reason="pool_within_target", K_pool=K, Nv_pool=Nv, Nv_post=Nv)
    mass = [float(w) + math.log(m) for w, m in zip(lw, mult)]
    counts = [0] * K
    ids = []
    distinct = draws = 0
    discarded = None
    for slot in range(1, 3 * Ns + 1):
        i = categorical(mass, float(event_uniforms(seed, DOMAIN_SIR_SLOT, event, slot, 1)[0]))
        draws = slot
        if distinct == Ns and counts[i] == 0:   # checked before keeping the hit, also on the last draw
            discarded = i
            break
        ids.append(i)
        distinct += counts[i] == 0
        counts[i] += 1
    return dict(selected_candidate=ids, multiplicity=counts, active=[i for i in range(K) if counts[i] > 0],
                common_log_weight=logsumexp(mass) - math.log(Nv), output_relative_log_weight=[0.0] * K,
                draw_count=draws, discarded_candidate=discarded,
                stop_reason="draw_limit" if discarded is None else "next_distinct", K_pool=K, Nv_pool=Nv,
                Nv_post=len(ids))


def aligned_weights(records):
    """``_aligned_weights`` (``ensemble.jl:26-30``)."""
    scale = max(r["weight_log_scale"] for r in records)
    return [r["relative_log_weight"] + (r["weight_log_scale"] - scale) for r in records], scale


def resampling_plan(records, scores, opts, statistics):
    """``_resampling_plan`` (``event.jl:1-16``): parent masses, LOO proposal
    probabilities, the mixture coefficient and the fresh-draw count M.
    ``statistics`` is the ensemble statistics of ``records`` (its ``eta_p``)."""
    relative, _ = aligned_weights(records)
    relative = np.asarray(relative)
    counts = np.asarray([r["count"] for r in records], float)
    mass = relative - relative.max() + np.log(counts)
    loo = loo_log_probabilities(mass, scores)
    p0 = np.asarray([r["log_p0"] for r in records], float)
    physical = np.asarray([r["physical_log_norm"] for r in records], float) - p0
    risk = mass + (physical - physical.max())
    selection = select_lambda(risk, loo - p0, opts.lambda_max, opts.lambda_tolerance)
    Ns = statistics["target_samples"]
    M = int(min(max(Ns - math.floor(statistics["eta_p"] * Ns), 0), Ns - 1))
    return dict(selection=selection, M=M, loo_log_probability=loo, loo_log_ratio=loo - p0,
                risk_log_amplitude_squared=risk, parent_log_mass=mass, pre_statistics=statistics)


def resample_fresh_count(plan, opts) -> int:
    """``_resample_fresh_count`` (``event.jl:17-20``)."""
    grow = opts.max_resample_sweep > 1 and plan["selection"]["lam"] < opts.lambda_threshold
    return max(1, plan["M"]) if grow else plan["M"]


def resample_stop(lam: float, sweep: int, opts) -> str:
    """``_resample_stop`` (``event.jl:21-25``)."""
    if lam >= opts.lambda_threshold:
        return "lambda_threshold"
    if sweep >= opts.max_resample_sweep:
        return "sweep_limit"
    return "continue"


class ScoreTable:
    """``ResamplingScores`` (``scores.jl:1-36``): configuration probabilities of
    one event, keyed by (member id, configuration column); member 0 is the
    beta0 Born distribution of the thermal PEPO."""

    def __init__(self):
        self.configurations = []
        self.columns = {}
        self.entries = []
        self.index = {}

    def columns_of(self, configurations):
        out = []
        for x in configurations:
            key = tuple(np.asarray(x).reshape(-1).tolist())
            j = self.columns.get(key)
            if j is None:
                self.configurations.append(np.asarray(x).copy())
                j = len(self.configurations)
                self.columns[key] = j
            out.append(j)
        return out

    def record(self, member_id, column, log_probability, max_environment_truncation=0.0, repairs=None,
               source="score"):
        key = (member_id, column)
        if key in self.index:
            return
        self.entries.append(dict(member_id=member_id, configuration_index=column, log_probability=log_probability,
                                 max_environment_truncation=max_environment_truncation,
                                 repairs=repairs or {}, source=source))
        self.index[key] = len(self.entries) - 1

    def get(self, member_id, column):
        return self.entries[self.index[(member_id, column)]]

    def matrix(self, member_ids, columns):
        return np.array([[self.get(i, j)["log_probability"] for j in columns] for i in member_ids])
