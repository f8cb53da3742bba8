"""``run_purification`` / ``run_stochastic`` over the device engine.

Restates the control flow of ``src/driver/run.jl:2-66,76-134``,
``src/driver/particles.jl:27-119`` and ``src/statistics/ensemble.jl``: the
same temperature grid, step schedule, particle weights, ensemble statistics
and result record (schema 2.7.0 field names).  Born draws take their
uniforms from ``sample_uniforms(seed, index, n)``, the explicit replacement
of the reference's ``sample_rng(seed, index)`` stream.  Annealed Born
resampling (``src/resample/event.jl``) runs when the ensemble's efficiency
falls below ``eta_th``, over the same ranks (scores, draws and fresh samples
on their owners, selected particles moved to their new owners); its math is
in ``resample.py``.  File output (JLD2, run.log) is not part of this engine.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np

from .config import (RunConfig, validate_config, temperature_nodes, measure_at, same_beta, parameter_dict)
from . import engine as eng

RESULT_SCHEMA_VERSION = "2.7.0"


def sample_uniforms(seed: int, index: int, n: int) -> np.ndarray:
    """The n uniforms of Born draw ``index`` (1-based) of run ``seed``."""
    if seed < 0 or index < 1:
        raise ValueError("invalid random stream identity")
    return np.random.default_rng([int(seed), int(index)]).random(n)


def step_schedule(start, target, delta_tau):
    """``_step_schedule`` (``particles.jl:55-64``)."""
    steps = []
    b = float(start)
    while not same_beta(b, target):
        if not target > b:
            raise ValueError("evolution requires increasing beta endpoints")
        b = min(target, b + 2 * delta_tau)
        if same_beta(b, target):
            b = float(target)
        steps.append(b)
    return steps


def ensemble_statistics(relative, multiplicity, energy, Ns, log_scale=0.0, nsites=1):
    """``ensemble_statistics`` (``src/statistics/ensemble.jl:8-25``)."""
    relative = np.asarray(relative, float)
    multiplicity = np.asarray(multiplicity, float)
    energy = np.asarray(energy, float)
    if not (len(relative) == len(multiplicity) == len(energy) > 0):
        raise ValueError("empty or inconsistent ensemble")
    if not (np.all(np.isfinite(relative)) and np.all(multiplicity > 0)):
        raise ValueError("invalid particle weights/counts")
    Nv = multiplicity.sum()
    pivot = relative.max()
    w = np.exp(relative - pivot)
    mass = multiplicity * w
    total = mass.sum()
    mu1 = total / Nv
    mu2 = float(np.sum(multiplicity * w ** 2) / Nv)
    eta = min(max(mu1 ** 2 / mu2, 1 / Nv), 1.0)

    def sem(f):
        return math.nan if Nv <= 1 else math.sqrt(max(0.0, float(np.sum(multiplicity * f ** 2)) / (Nv * (Nv - 1))))

    measured = bool(np.all(np.isfinite(energy)))
    E = float(np.sum(mass * energy) / total) if measured else math.nan
    Eerr = sem(w * (energy - E) / mu1) if measured else math.nan
    return dict(energy_total=nsites * E, energy_per_site=E, energy_per_site_error=Eerr,
                lnZ=log_scale + pivot + math.log(mu1), lnZ_error=sem((w - mu1) / mu1), eta=eta,
                eta_error=sem((2 * mu1 / mu2) * (w - mu1) - (mu1 ** 2 / mu2 ** 2) * (w ** 2 - mu2)),
                ESS=Nv * eta,
                eta_p=min(max(total ** 2 / (Ns * float(np.sum(mass ** 2))), 1 / Ns), len(relative) / Ns),
                target_samples=Ns, virtual_samples=Nv, representatives=len(relative))


def group_configurations(configurations):
    """``_group_configurations`` (``src/resample/selection.jl:122-140``), 1-based draws."""
    first, mult, d2g = [], [], []
    lookup = {}
    for d, x in enumerate(configurations, start=1):
        key = tuple(np.asarray(x).reshape(-1).tolist())
        j = lookup.get(key)
        if j is None:
            first.append(d)
            mult.append(0)
            j = len(first)
            lookup[key] = j
        mult[j - 1] += 1
        d2g.append(j)
    return dict(first_draw=first, multiplicity=mult, draw_to_group=d2g)


@dataclass
class ThermalCheckpoint:
    """Thermal PEPO at beta0 plus preparation records (``src/io/run_output.jl:4-11``)."""
    state: eng.DeviceState
    preparation: dict
    purification: list
    history: list
    run_id: str


@dataclass
class Particle:
    """A Born sample with its normalisation and estimator weight (``particles.jl:2-25``)."""
    id: int
    count: int
    configuration: np.ndarray
    state: eng.DeviceState
    log_p0: float
    log_q_proposal: float
    relative_log_weight: float
    weight_log_scale: float
    physical_log_norm: float
    tensor_log_norm: float
    energy_total: float
    energy_per_site: float
    magnetization: float
    max_state_truncation: float = 0.0
    max_environment_truncation: float = 0.0
    max_boundary_entropy: float = math.nan
    time_seconds: float = 0.0
    measurement_seconds: float = 0.0
    generation: int = 0
    sample_index: int = 0
    seed: int = 0


class DeviceOps:
    """The hot-path operations the drivers call, on the device engine."""

    def sampling_cache(self, state, method, kind="auxiliary"):
        return eng.SamplingCache(state, method, kind)

    def sample(self, cache, uniforms):
        return eng.sample_configuration(cache, uniforms=uniforms)

    def probability(self, cache, configuration):
        return eng.sample_configuration(cache, configuration=configuration)

    def probability_batch(self, cache, configurations):
        lps, reps = eng.sample_probability_batch(cache, np.stack([np.asarray(x) for x in configurations]))
        return [dict(r, log_probability=float(lp)) for lp, r in zip(lps, reps)]

    # a particle's state between ranks (a resampling event moves selected particles)
    def export_state(self, state):
        sites, dims = state.download()
        return dict(sites=sites, dims=np.asarray(dims), is_pepo=state.is_pepo, beta=state.beta,
                    log_amplitude=state.log_amplitude)

    def import_state(self, blob, like):
        return like.engine.upload_state(blob["sites"], blob["dims"], blob["is_pepo"], beta=blob["beta"],
                                        log_amplitude=blob["log_amplitude"])

    def state_from(self, blob, c: RunConfig, engine=None):
        """An exported state on a new engine for ``c`` (a checkpoint being loaded)."""
        e = engine or eng.Engine.from_config(c)
        return e.upload_state(blob["sites"], blob["dims"], blob["is_pepo"], beta=blob["beta"],
                              log_amplitude=blob["log_amplitude"])

    def project(self, state, configuration):
        return eng.project_configuration(state, configuration)

    def measure_energy(self, state, method):
        return eng.measure_energy(state, method)

    def lognorm(self, state, method):
        return eng.lognorm(state, method)

    def evolution_step(self, state, delta, D, method, space):
        return eng.evolution_step(state, delta, D, method, space)

    # batched forms: one library call over many samples (sps_*_batch)
    def sample_batch(self, cache, uniforms):
        cfgs, lps, reps = eng.sample_batch(cache, uniforms, reports=True)
        return [dict(configuration=c, log_probability=float(lp), **r) for c, lp, r in zip(cfgs, lps, reps)]

    def project_batch(self, state, configurations):
        states, ln = eng.project_batch(state, configurations)
        return list(zip(states, ln))

    def measure_energy_batch(self, states, method):
        return eng.measure_energy_batch(states, method)

    def lognorm_batch(self, states, method):
        return eng.lognorm_batch(states, method)

    def evolution_step_batch(self, states, deltas, D, method, space):
        return eng.evolution_step_batch(states, deltas, D, method, space)


DEVICE_OPS = DeviceOps()


def _batched(ops, name, single, items, *args):
    """ops.<name>_batch(items, *args) when the ops provide it, else the single
    operation item by item (the ops of a test double may define only those)."""
    f = getattr(ops, name + "_batch", None)
    if f is not None:
        return list(f(items, *args))
    return [single(x, *args) for x in items]


def _observe_batch(states, c: RunConfig, energy: bool, ops=DEVICE_OPS):
    """``_observe`` of many states in one call; the elapsed time is shared equally."""
    t = time.perf_counter()
    method = c.boundary("measurement")
    if energy:
        ms = _batched(ops, "measure_energy", ops.measure_energy, states, method)
    else:
        ms = _batched(ops, "lognorm", ops.lognorm, states, method)
        for m in ms:
            m.update(energy_total=math.nan, energy_per_site=math.nan, magnetization=math.nan)
    dt = (time.perf_counter() - t) / max(1, len(states))
    for m in ms:
        m["measurement_seconds"] = dt
    return ms


def _evolve_batch(states, c: RunConfig, steps, D, space, ops=DEVICE_OPS):
    """``_evolve!`` (``particles.jl:66-85``) of many states over the same beta
    schedule: one batched evolution step per beta; the elapsed time is shared
    equally."""
    n = len(states)
    out = [dict(time_seconds=0.0, max_state_truncation=0.0, max_environment_truncation=0.0,
                max_boundary_entropy=0.0 if (c.record_boundary_entropy and steps) else math.nan,
                normalization=0.0) for _ in range(n)]
    single = getattr(ops, "evolution_step_batch", None)
    for beta in steps:
        t = time.perf_counter()
        deltas = [(beta - s.beta) / 2 for s in states]
        if single is not None:
            reps = single(states, deltas, D, c.boundary("environment"), space)
        else:
            reps = [ops.evolution_step(s, d, D, c.boundary("environment"), space) for s, d in zip(states, deltas)]
        elapsed = (time.perf_counter() - t) / max(1, n)
        for s, r, o in zip(states, reps, out):
            s.beta = beta
            o["normalization"] += r["log_normalization_sum"]
            o["time_seconds"] += elapsed
            o["max_state_truncation"] = max(o["max_state_truncation"], r["max_state_truncation"])
            o["max_environment_truncation"] = max(o["max_environment_truncation"], r["max_environment_truncation"])
            o["max_boundary_entropy"] = max(o["max_boundary_entropy"], r["max_boundary_entropy"])
    return out


def _observe(state, c: RunConfig, energy: bool, ops=DEVICE_OPS):
    """``_observe`` (``particles.jl:35-40``)."""
    t = time.perf_counter()
    if energy:
        m = ops.measure_energy(state, c.boundary("measurement"))
    else:
        m = ops.lognorm(state, c.boundary("measurement"))
        m.update(energy_total=math.nan, energy_per_site=math.nan, magnetization=math.nan)
    m["measurement_seconds"] = time.perf_counter() - t
    return m


def _evolve(state, c: RunConfig, steps, D, space, on_step=None, ops=DEVICE_OPS):
    """``_evolve!`` (``particles.jl:66-85``)."""
    total = maxstate = maxenv = normalization = 0.0
    maxent = 0.0 if (c.record_boundary_entropy and steps) else math.nan
    for beta in steps:
        t = time.perf_counter()
        r = ops.evolution_step(state, (beta - state.beta) / 2, D, c.boundary("environment"), space)
        elapsed = time.perf_counter() - t
        state.beta = beta
        normalization += r["log_normalization_sum"]
        total += elapsed
        maxstate = max(maxstate, r["max_state_truncation"])
        maxenv = max(maxenv, r["max_environment_truncation"])
        maxent = max(maxent, r["max_boundary_entropy"])
        if on_step:
            on_step(dict(r, beta=beta, time_seconds=elapsed))
    return dict(time_seconds=total, max_state_truncation=maxstate, max_environment_truncation=maxenv,
                max_boundary_entropy=maxent, normalization=normalization)


def run_purification(c: RunConfig, engine: eng.Engine | None = None, ops=None,
                     identity=None) -> ThermalCheckpoint:
    """Prepare the beta0 thermal PEPO (``run.jl:2-43``)."""
    validate_config(c)
    ops = ops or DEVICE_OPS
    if identity is None:
        e = engine or eng.Engine.from_config(c)
        state = e.identity_pepo()
        initial = eng.normalize_state(state)
    else:
        state, initial = identity()
    history = [dict(phase="initialization", beta=0.0, normalizations=list(initial))]
    rows = []
    for beta in [b for b in temperature_nodes(c) if b <= c.beta0]:
        steps = step_schedule(state.beta, beta, c.delta_tau_pur)
        rep = _evolve(state, c, steps, c.D_pur, c.bond_space_pur, on_step=history.append, ops=ops)
        m = _observe(state, c, measure_at(c, beta), ops)
        rows.append(dict(beta=beta, source="purification", energy_total=m["energy_total"],
                         energy_per_site=m["energy_per_site"],
                         energy_per_site_error=0.0 if measure_at(c, beta) else math.nan,
                         lnZ=m["log_norm"], lnZ_error=0.0, eta=math.nan, eta_error=math.nan,
                         magnetization=m["magnetization"],
                         max_state_truncation=rep["max_state_truncation"],
                         max_environment_truncation=max(rep["max_environment_truncation"],
                                                        m["max_environment_truncation"]),
                         max_boundary_entropy=rep["max_boundary_entropy"],
                         time_seconds=rep["time_seconds"], measurement_seconds=m["measurement_seconds"]))
    return ThermalCheckpoint(state, parameter_dict(c), rows, history, f"run-{time.time_ns()}")


def _particle_record(p: Particle):
    """``_particle_scalar`` (``particles.jl:103-115``)."""
    return dict(id=p.id, generation=p.generation, sample_index=p.sample_index, seed=p.seed, count=p.count,
                configuration=p.configuration.copy(), owner=0, beta=p.state.beta, log_p0=p.log_p0,
                log_q_proposal=p.log_q_proposal, relative_log_weight=p.relative_log_weight,
                weight_log_scale=p.weight_log_scale, log_weight=p.weight_log_scale + p.relative_log_weight,
                physical_log_norm=p.physical_log_norm, log_amplitude=p.state.log_amplitude,
                energy_total=p.energy_total, energy_per_site=p.energy_per_site, magnetization=p.magnetization,
                max_state_truncation=p.max_state_truncation,
                max_environment_truncation=p.max_environment_truncation,
                max_boundary_entropy=p.max_boundary_entropy, time_seconds=p.time_seconds,
                measurement_seconds=p.measurement_seconds)


def _statistics(records, Ns, nsites):
    """``_statistics`` (``ensemble.jl:31-40``)."""
    scale = max(r["weight_log_scale"] for r in records)
    rel = [r["relative_log_weight"] + (r["weight_log_scale"] - scale) for r in records]
    s = ensemble_statistics(rel, [r["count"] for r in records], [r["energy_per_site"] for r in records], Ns,
                            log_scale=scale, nsites=nsites)
    s.update(beta=records[0]["beta"],
             max_state_truncation=max(r["max_state_truncation"] for r in records),
             max_environment_truncation=max(r["max_environment_truncation"] for r in records),
             max_boundary_entropy=max(r["max_boundary_entropy"] for r in records),
             distinct_configurations=len({tuple(np.asarray(r["configuration"]).reshape(-1)) for r in records}))
    mags = [r["magnetization"] for r in records]
    if all(math.isfinite(x) for x in mags):
        w = np.exp(np.asarray(rel) - max(rel)) * np.asarray([r["count"] for r in records])
        s["magnetization"] = float(np.sum(w * np.asarray(mags)) / np.sum(w))
    else:
        s["magnetization"] = math.nan
    return s


def _new_particles(checkpoint, c: RunConfig, items, energy: bool, ops=DEVICE_OPS):
    """``_new_particle`` (``particles.jl:42-52``) for many configurations at once:
    projection of the beta0 PEPO, one observation, estimator weight
    log_norm - log_q.  ``items``: dicts with id, count, configuration, log_p0,
    log_q, sampling_error and generation."""
    if not items:
        return []
    cfgs = [np.asarray(it["configuration"]) for it in items]
    if hasattr(ops, "project_batch"):
        projected = ops.project_batch(checkpoint.state, np.stack(cfgs))
    else:
        projected = [ops.project(checkpoint.state, x) for x in cfgs]
    states = [p[0] for p in projected]
    obs = _observe_batch(states, c, energy, ops)
    out = []
    for it, state, m in zip(items, states, obs):
        out.append(Particle(id=it["id"], count=it["count"], configuration=np.asarray(it["configuration"]),
                            state=state, log_p0=it["log_p0"], log_q_proposal=it["log_q"],
                            relative_log_weight=m["log_norm"] - it["log_q"], weight_log_scale=0.0,
                            physical_log_norm=m["log_norm"], tensor_log_norm=m["tensor_log_norm"],
                            energy_total=m["energy_total"], energy_per_site=m["energy_per_site"],
                            magnetization=m["magnetization"],
                            max_environment_truncation=max(it["sampling_error"], m["max_environment_truncation"]),
                            measurement_seconds=m["measurement_seconds"], generation=it.get("generation", 0),
                            sample_index=it["id"], seed=c.seed))
    return out


def _advance_particles(particles, c: RunConfig, steps, energy: bool, ops=DEVICE_OPS):
    """``_advance_particle!`` (``particles.jl:86-102``) for every particle, batched per step."""
    if not particles:
        return
    states = [p.state for p in particles]
    reps = _evolve_batch(states, c, steps, c.D_peps, c.bond_space_peps, ops=ops)
    obs = _observe_batch(states, c, energy, ops)
    for p, rep, m in zip(particles, reps, obs):
        old = p.tensor_log_norm
        p.relative_log_weight += 2 * rep["normalization"] + (m["tensor_log_norm"] - old)
        p.physical_log_norm = m["log_norm"]
        p.tensor_log_norm = m["tensor_log_norm"]
        p.energy_total = m["energy_total"]
        p.energy_per_site = m["energy_per_site"]
        p.magnetization = m["magnetization"]
        p.max_state_truncation = rep["max_state_truncation"]
        p.max_environment_truncation = max(rep["max_environment_truncation"], m["max_environment_truncation"])
        p.max_boundary_entropy = rep["max_boundary_entropy"]
        p.time_seconds = rep["time_seconds"]
        p.measurement_seconds = m["measurement_seconds"]


def run_stochastic(c: RunConfig, checkpoint: ThermalCheckpoint | None = None, uniforms_fn=None, execution=None,
                   ops=None, checkpoint_path=None):
    """Draw Born samples from the beta0 checkpoint and evolve the weighted ensemble (``run.jl:76-134``).

    ``execution`` distributes the work like the reference's MPI backend
    (``ext/StoPEPSMPIExt.jl``): draws round-robin by index, unique
    configurations by representative position, scalar records gathered at
    every node; the default runs serially.  Rank 0 returns the result record
    (``observables``: curve, purification, samples; ``diagnostics``: Born
    draws and grouping; ``metadata``; ``parameters``); other ranks return None.
    """
    from .parallel import SerialExecution
    e = execution or SerialExecution()
    ops = ops or DEVICE_OPS
    e.phase(lambda: validate_config(c))
    e.check_arguments(repr(parameter_dict(c)))
    if checkpoint is None:
        # the checkpoint from disk (run.jl:79-87): every rank loads it
        if checkpoint_path is None:
            raise ValueError("supply a checkpoint or checkpoint_path")
        from .checkpoint import load_checkpoint
        checkpoint = e.phase(lambda: load_checkpoint(checkpoint_path, c, ops))

    def check_checkpoint():
        if not same_beta(checkpoint.state.beta, c.beta0):
            raise ValueError("checkpoint model, lattice or beta0 mismatch")

    e.phase(check_checkpoint)
    L = c.lattice.Lx * c.lattice.Ly
    if uniforms_fn is None:
        uniforms_fn = lambda i: sample_uniforms(c.seed, i, L)
    rank, nprocs = e.rank(), e.nprocs()

    cache = e.phase(lambda: ops.sampling_cache(checkpoint.state, c.boundary("sampling")))

    def local_draws():
        idx = [i for i in range(1, c.Ns + 1) if (i - 1) % nprocs == rank]
        if not idx:
            return []
        if hasattr(ops, "sample_batch"):   # every local draw in one call
            out = [dict(d) for d in ops.sample_batch(cache, np.stack([uniforms_fn(i) for i in idx]))]
        else:
            out = [dict(ops.sample(cache, uniforms_fn(i))) for i in idx]
        for d, i in zip(out, idx):
            d["index"] = i
        return out

    draws = sorted([d for part in e.gather(e.phase(local_draws)) for d in part], key=lambda d: d["index"])
    grouping = group_configurations([d["configuration"] for d in draws])

    def local_particles():
        # _representative_owner (src/driver/execution.jl:34): unique configuration u on rank (u-1) % nprocs
        items = [dict(id=i, count=grouping["multiplicity"][u - 1], configuration=draws[i - 1]["configuration"],
                      log_p0=draws[i - 1]["log_probability"], log_q=draws[i - 1]["log_probability"],
                      sampling_error=draws[i - 1]["max_environment_truncation"])
                 for u, i in enumerate(grouping["first_draw"], start=1) if (u - 1) % nprocs == rank]
        return _new_particles(checkpoint, c, items, measure_at(c, c.beta0), ops)

    particles = e.phase(local_particles)
    curve = [r for r in checkpoint.purification if r["beta"] < c.beta0 and not same_beta(r["beta"], c.beta0)]
    samples, events, replay_rows = [], [], []
    replay = []   # the evolution history: (beta, steps) per output node, replayed by fresh samples
    event, next_sample_id = 0, c.Ns + 1
    nodes = [b for b in temperature_nodes(c) if b >= c.beta0]
    for node, beta in enumerate(nodes):
        steps = [] if node == 0 else step_schedule(nodes[node - 1], beta, c.delta_tau_peps)
        replay.append(dict(beta=beta, steps=list(steps)))
        if node > 0:
            e.phase(lambda: _advance_particles(particles, c, steps, measure_at(c, beta), ops))
        local_records = e.phase(lambda: [dict(_particle_record(p), owner=rank) for p in particles])
        records = sorted([r for part in e.gather(local_records) for r in part], key=lambda r: r["id"])
        stats = _statistics(records, c.Ns, L)
        stats.update(source="sampling",
                     time_seconds=max(e.gather(sum(p.time_seconds for p in particles))))
        if c.resampling.enabled and stats["eta"] < c.resampling.eta_th:
            event += 1
            particles, records, stats, next_sample_id, audit = _resample(
                particles, records, checkpoint, c, cache, replay, event, next_sample_id, ops, e)
            events.append(audit)
            replay_rows.extend(audit.pop("replay_rows"))
        curve.append(stats)
        samples.extend(records)
    if rank != 0:
        return None
    return {"schema_version": RESULT_SCHEMA_VERSION, "method": "stoPEPS",
            "parameters": parameter_dict(c), "model": parameter_dict(c)["model"],
            "observables": {"curve": curve, "purification": list(checkpoint.purification),
                            "samples": samples, "replay": replay_rows},
            "diagnostics": {"born_draws": draws, "born_grouping": grouping, "events": events,
                            "history": list(checkpoint.history)},
            "metadata": {"run_id": checkpoint.run_id, "stage": "stochastic", "complete": True,
                         "mpi_size": nprocs, "restart_supported": False,
                         "uncertainty": "conditional_particle_delta_method; shared_history_scale_fixed"}}


# ---------------------------------------------------------------------------
# annealed Born resampling (src/resample/event.jl, scores.jl)
# ---------------------------------------------------------------------------
_REPAIR_KEYS = ("metric_repairs", "zero_proposals", "min_relative_eigenvalue")


def _score(memo, caches, member_ids, configurations, ops, e):
    """``_score_configurations!`` (``scores.jl:38-71``): the probabilities of
    ``configurations`` under each member's cache that the table does not hold
    yet.  The beta0 column j is scored on rank (j-1) % nprocs, a member's on
    the rank holding its cache; one batched call per member, then every rank
    records every entry (ordered by member and column).  Returns the member
    ids and the configurations' columns."""
    columns = memo.columns_of(configurations)
    unique = list(dict.fromkeys(columns))
    rank, nprocs = e.rank(), e.nprocs()

    def local():
        out = []
        for mid in member_ids:
            if mid == 0:
                todo = [j for j in unique if (j - 1) % nprocs == rank]
            elif mid in caches:
                todo = list(unique)
            else:
                continue
            todo = [j for j in todo if (mid, j) not in memo.index]
            if not todo:
                continue
            cfgs = [memo.configurations[j - 1] for j in todo]
            if hasattr(ops, "probability_batch"):
                res = ops.probability_batch(caches[mid], cfgs)
            else:
                res = [ops.probability(caches[mid], x) for x in cfgs]
            for j, r in zip(todo, res):
                out.append(dict(member_id=mid, column=j, log_probability=float(r["log_probability"]),
                                max_environment_truncation=r.get("max_environment_truncation", 0.0),
                                repairs={k: r[k] for k in _REPAIR_KEYS if k in r}))
        return out

    parts = e.gather(e.phase(local))
    for r in sorted([r for p in parts for r in p], key=lambda r: (r["member_id"], r["column"])):
        memo.record(r["member_id"], r["column"], r["log_probability"], r["max_environment_truncation"],
                    r["repairs"])

    def check():
        for mid in member_ids:
            for j in unique:
                if (mid, j) not in memo.index:
                    raise RuntimeError("missing proposal scores")
    e.phase(check)
    return dict(member_ids=list(member_ids), configuration_indices=columns)


def _evaluate_resampling(memo, caches, particles, records, c: RunConfig, ops, e, after_sweep):
    """``_evaluate_resampling!`` (``event.jl:27-43``): a physical-kind proposal
    cache per local particle, the leave-one-out score matrix, and the plan
    (made on rank 0, broadcast)."""
    from . import resample as rs
    t = time.perf_counter()

    def build():
        for p in particles:
            if p.id not in caches:
                caches[p.id] = ops.sampling_cache(p.state, c.boundary("proposal"), "physical")
    e.phase(build)
    ref = _score(memo, caches, [r["id"] for r in records], [r["configuration"] for r in records], ops, e)
    plan = e.broadcast(lambda: rs.resampling_plan(
        records, memo.matrix(ref["member_ids"], ref["configuration_indices"]), c.resampling,
        _statistics(records, c.Ns, c.lattice.Lx * c.lattice.Ly)))
    seconds = max(e.gather(time.perf_counter() - t))
    return dict(after_sweep=after_sweep, plan=plan, score_reference=ref, loo_seconds=seconds)


def _draw_resampling_batch(memo, caches, records, plan, M, c: RunConfig, event, sweep, ops, e):
    """``_draw_resampling_batch!`` (``event.jl:114-174``): M fresh draws from the
    mixture proposal (member 0, the beta0 Born distribution, with probability
    1 - lambda, else a pool member by its parent mass), each on the rank that
    owns its component (member 0: draw d on rank (d-1) % nprocs); their
    grouping, the baseline and mixture scores of the distinct configurations
    and their proposal log-probabilities log q (made on rank 0, broadcast)."""
    from . import resample as rs
    lam = plan["selection"]["lam"]
    L = c.lattice.Lx * c.lattice.Ly
    rank, nprocs = e.rank(), e.nprocs()
    slots = [(sweep - 1) * c.Ns + d for d in range(1, M + 1)]

    def choose():
        out = []
        for slot in slots:
            u = rs.event_uniforms(c.seed, rs.DOMAIN_MIXTURE, event, slot, 2)
            out.append(rs.categorical(list(plan["parent_log_mass"]), u[1]) + 1 if u[0] < lam else 0)
        return out
    members = e.broadcast(choose)

    def local_draws():
        out = []
        for d, (slot, member) in enumerate(zip(slots, members), start=1):
            owner = (d - 1) % nprocs if member == 0 else records[member - 1]["owner"]
            if owner != rank:
                continue
            mid = 0 if member == 0 else records[member - 1]["id"]
            r = ops.sample(caches[mid], rs.event_uniforms(c.seed, rs.DOMAIN_FRESH, event, slot, L))
            out.append(dict(index=d, slot=slot, member=member, member_id=mid,
                            configuration=np.asarray(r["configuration"]),
                            selected_log_probability=float(r["log_probability"]),
                            max_environment_truncation=r.get("max_environment_truncation", 0.0),
                            repairs={k: r[k] for k in _REPAIR_KEYS if k in r}))
        return out
    draws = sorted([d for p in e.gather(e.phase(local_draws)) for d in p], key=lambda d: d["index"])
    # _seed_draw_scores! (scores.jl:73-87): a draw has evaluated its own component
    for d, col in zip(draws, memo.columns_of([d["configuration"] for d in draws])):
        memo.record(d["member_id"], col, d["selected_log_probability"], d["max_environment_truncation"],
                    d["repairs"], source="draw")
    grouping = group_configurations([d["configuration"] for d in draws])
    configurations = [draws[i - 1]["configuration"] for i in grouping["first_draw"]]
    baseline = _score(memo, caches, [0], configurations, ops, e)
    scored_ref = None if lam == 0 else _score(memo, caches, [r["id"] for r in records], configurations, ops, e)

    def make_proposals():
        norm = rs.logsumexp(plan["parent_log_mass"])
        out = []
        for col in baseline["configuration_indices"]:
            p0 = memo.get(0, col)
            scored = [] if scored_ref is None else [memo.get(i, col) for i in scored_ref["member_ids"]]
            pr = None if scored_ref is None else rs.logsumexp(
                [m + s["log_probability"] for m, s in zip(plan["parent_log_mass"], scored)]) - norm
            q = rs.mixture_log_probability(p0["log_probability"], pr, lam)
            err = max([p0["max_environment_truncation"]] + [s["max_environment_truncation"] for s in scored])
            out.append(dict(log_p0=p0["log_probability"], log_pr=pr, log_q=q, max_environment_truncation=err))
        return out
    proposals = e.broadcast(make_proposals)
    for i, d in enumerate(draws):
        g = proposals[grouping["draw_to_group"][i] - 1]
        d["log_probability"] = g["log_q"]
        d["max_environment_truncation"] = max(d["max_environment_truncation"], g["max_environment_truncation"])
    return dict(members=members, draws=draws, grouping=grouping, configurations=configurations, proposals=proposals,
                baseline_reference=baseline, score_reference=scored_ref)


def _global_records(particles, e):
    """``_global_particles`` (``particles.jl:116-119``): every rank's particle
    records, owner set, ordered by id."""
    rank = e.rank()
    local = e.phase(lambda: [dict(_particle_record(p), owner=rank) for p in particles])
    return sorted([r for part in e.gather(local) for r in part], key=lambda r: r["id"])


def _replay_fresh(fresh, replay, c: RunConfig, event, sweep, ops, e):
    """``_replay_fresh!`` (``event.jl:79-112``): the local fresh samples re-evolved
    through the saved step endpoints, observed at every output node (energy
    where the node is measured); one statistics row of all ranks' fresh
    samples per node."""
    rows = []
    records = []
    for node, segment in enumerate(replay):
        if node > 0:
            e.phase(lambda: _advance_particles(fresh, c, segment["steps"],
                                               node == len(replay) - 1 and measure_at(c, segment["beta"]), ops))
        records = _global_records(fresh, e)
        seconds = max(e.gather(sum(p.time_seconds for p in fresh)))
        if records:
            stats = _statistics(records, sum(r["count"] for r in records), c.lattice.Lx * c.lattice.Ly)
            stats.update(event=event, sweep=sweep, time_seconds=seconds, source="fresh_replay")
            rows.append(dict(event=event, sweep=sweep, statistics=stats, samples=records))
    return records, rows


def _redistribute(pool_particles, pool, selection, ops, e, like):
    """``_redistribute`` (``execution.jl:28-31``, ``ext/StoPEPSMPIExt.jl:32-51``):
    the selected pool members, the k-th of them (in selection order) to rank
    k % nprocs, with the selection's counts and weights.  A member held by
    another rank moves with its state exported through the ops."""
    rank, nprocs = e.rank(), e.nprocs()
    held = {p.id: p for p in pool_particles}
    nxt, outgoing = [], []
    for position, i in enumerate(selection["active"]):
        source, dest = pool[i]["owner"], position % nprocs
        if rank == source and source == dest:
            nxt.append((i, held[pool[i]["id"]]))
        elif rank == source:
            p = held[pool[i]["id"]]
            blob = dict(p.__dict__)
            blob["state"] = ops.export_state(p.state)
            outgoing.append((dest, i, blob))
    for part in e.gather(outgoing):
        for dest, i, blob in part:
            if dest == rank:
                blob = dict(blob)
                blob["state"] = ops.import_state(blob["state"], like)
                nxt.append((i, Particle(**blob)))
    out = []
    for i, p in sorted(nxt, key=lambda t: selection["active"].index(t[0])):
        p.count = selection["multiplicity"][i]
        p.relative_log_weight = selection["output_relative_log_weight"][i]
        p.weight_log_scale = selection["common_log_weight"]
        out.append(p)
    return out


def _resample(particles, records, checkpoint, c: RunConfig, baseline_cache, replay, event, next_sample_id, ops,
              e=None):
    """``_resample!`` (``event.jl:176-253``): one annealed Born resampling event.

    Leave-one-out plan, then up to ``max_resample_sweep`` sweeps of fresh draws
    from the mixture proposal, each sweep's distinct configurations projected
    from the beta0 PEPO (the u-th on rank (u-1) % nprocs, the representative
    owner of ``execution.jl:34``), replayed to the current beta and added to
    the pool, with a new plan after every sweep that does not stop; finally
    SIR selection of Ns distinct representatives from the pool with equal
    weights, moved to their new owners.  ``particles`` are this rank's,
    ``records`` every rank's.  Returns this rank's new particles, every
    rank's records and their statistics, the next free sample id and the
    event's audit record."""
    from . import resample as rs
    from .parallel import SerialExecution
    e = e or SerialExecution()
    rank, nprocs = e.rank(), e.nprocs()
    started = time.perf_counter()
    beta = replay[-1]["beta"]
    interval_seconds = max(e.gather(sum(p.time_seconds for p in particles)))
    memo = rs.ScoreTable()
    caches = {0: baseline_cache}
    evaluations, sweeps, replay_rows = [], [], []
    evaluation = _evaluate_resampling(memo, caches, particles, records, c, ops, e, 0)
    evaluations.append(evaluation)
    plan = evaluation["plan"]
    M = rs.resample_fresh_count(plan, c.resampling)
    pool_particles = list(particles)
    pool_records = list(records)
    all_fresh = []
    stop_reason = "continue"
    proposal_seconds = replay_seconds = 0.0
    for sweep in range(1, c.resampling.max_resample_sweep + 1):
        t = time.perf_counter()
        batch = _draw_resampling_batch(memo, caches, pool_records, plan, M, c, event, sweep, ops, e)
        proposal_time = max(e.gather(time.perf_counter() - t))
        proposal_seconds += proposal_time
        lam = plan["selection"]["lam"]
        stop_reason = "no_fresh_draws" if M == 0 else rs.resample_stop(lam, sweep, c.resampling)
        if stop_reason != "continue":
            caches.clear()   # proposal environments are released before the last replay
        first_id = next_sample_id
        next_sample_id += c.Ns
        t = time.perf_counter()
        items = [dict(id=first_id + d - 1, count=batch["grouping"]["multiplicity"][u], generation=event,
                      configuration=batch["configurations"][u], log_p0=batch["proposals"][u]["log_p0"],
                      log_q=batch["proposals"][u]["log_q"],
                      sampling_error=batch["proposals"][u]["max_environment_truncation"])
                 for u, d in enumerate(batch["grouping"]["first_draw"]) if u % nprocs == rank]
        fresh = e.phase(lambda: _new_particles(checkpoint, c, items, len(replay) == 1 and measure_at(c, beta), ops))
        fresh_records, rows = ([], []) if M == 0 else _replay_fresh(fresh, replay, c, event, sweep, ops, e)
        replay_rows.extend(rows)
        replay_time = max(e.gather(time.perf_counter() - t))
        replay_seconds += replay_time
        pool_particles.extend(fresh)
        all_fresh.extend(fresh_records)
        pool_records = list(records) + all_fresh
        sweeps.append(dict(sweep=sweep, evaluation=len(evaluations), lam=lam, M=M, members=batch["members"],
                           draws=batch["draws"], grouping=batch["grouping"], proposals=batch["proposals"],
                           fresh_ids=[r["id"] for r in fresh_records], pool_representatives=len(pool_records),
                           pool_virtual_samples=sum(r["count"] for r in pool_records),
                           timing=dict(proposal_seconds=proposal_time, replay_seconds=replay_time)))
        if stop_reason != "continue":
            break
        evaluation = _evaluate_resampling(memo, caches, pool_particles, pool_records, c, ops, e, sweep)
        evaluations.append(evaluation)
        plan = evaluation["plan"]
        if plan["selection"]["lam"] >= c.resampling.lambda_threshold:
            stop_reason = "lambda_threshold"
            break
    caches.clear()
    pool = list(records) + all_fresh

    def pool_selection():
        """``_pool_selection`` (``event.jl:69-77``)."""
        relative, scale = rs.aligned_weights(pool)
        pivot = max(relative)
        sel = rs.sir_select_until_unique([v - pivot for v in relative], [r["count"] for r in pool], c.Ns,
                                         c.seed, event)
        sel.update(common_log_weight=scale + pivot + sel["common_log_weight"],
                   pool_statistics=_statistics(pool, c.Ns, c.lattice.Lx * c.lattice.Ly))
        return sel
    selection = e.broadcast(pool_selection)
    nxt = _redistribute(pool_particles, pool, selection, ops, e, checkpoint.state)
    post = _global_records(nxt, e)
    stats = _statistics(post, c.Ns, c.lattice.Lx * c.lattice.Ly)
    stats.update(source="sampling", time_seconds=interval_seconds)
    audit = dict(event=event, beta=beta, M=M,
                 lambda_evaluations=[dict(after_sweep=v["after_sweep"], lam=v["plan"]["selection"]["lam"],
                                          selection=v["plan"]["selection"], M=v["plan"]["M"],
                                          loo_log_probability=v["plan"]["loo_log_probability"].tolist(),
                                          parent_log_mass=v["plan"]["parent_log_mass"].tolist(),
                                          loo_seconds=v["loo_seconds"]) for v in evaluations],
                 sweeps=sweeps, stop_reason=stop_reason,
                 score_table=dict(configurations=memo.configurations,
                                  entries=sorted(memo.entries, key=lambda r: (r["member_id"],
                                                                              r["configuration_index"]))),
                 pre=list(records), fresh=all_fresh, selection=selection, post=post, post_statistics=stats,
                 accepted=True, proposal="finite_chi_psd_sequential_basis",
                 timing=dict(loo_seconds=sum(v["loo_seconds"] for v in evaluations),
                             proposal_seconds=proposal_seconds, replay_seconds=replay_seconds,
                             total_seconds=time.perf_counter() - started),
                 replay_rows=replay_rows)
    return nxt, post, stats, next_sample_id, audit
