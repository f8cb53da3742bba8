"""Drivers, weights and ensemble statistics for the CPU oracle.

TEST INFRASTRUCTURE ONLY (see ``oracle/z2.py``).

Restates ``src/driver/particles.jl:27-102``, ``src/driver/run.jl:2-66,76-127``
(resampling disabled), ``src/driver/config.jl:63-76`` and
``src/statistics/ensemble.jl``.  Born draws take uniforms from
``sample_uniforms(seed, index, n)`` in place of ``sample_rng``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .z2 import EPS
from . import boundary as bm
from . import full_update as fu
from . import diagonal as dg
from . import sampling as sp
from .model import TFIM, identity_pepo, normalize_state


@dataclass
class RunConfig:
    """The fields of ``RunConfig`` (``config.jl:28-62``) this path reads."""
    Lx: int = 2
    Ly: int = 2
    J: float = 1.0
    h: float = 0.7
    fields: tuple | None = None   # per-site transverse fields (extension; x + y*Lx order)
    beta0: float = 0.1
    beta_log: list = field(default_factory=lambda: [0.0, 0.05, 0.1, 0.15, 0.2, 0.25, 0.3])
    beta_measure: list = field(default_factory=lambda: [0.0, 0.1, 0.2, 0.3])
    delta_tau_pur: float = 0.025
    delta_tau_peps: float = 0.025
    D_pur: int = 4
    D_peps: int = 4
    bond_space_pur: tuple | None = None
    bond_space_peps: tuple | None = None
    chi_environment: int = 32
    chi_sampling: int | None = None
    chi_measurement: int | None = None
    environment_space: tuple | None = None
    sampling_space: tuple | None = None
    measurement_space: tuple | None = None
    trotter_order: int = 2
    update: fu.FullUpdate = field(default_factory=fu.FullUpdate)
    record_boundary_entropy: bool = True
    Ns: int = 16
    seed: int = 20260924
    diagonal: bool = False   # contraction = BoundaryMPSDiagonal (src/contraction/diagonal_mps.jl)

    def boundary(self, role):
        chi = getattr(self, "chi_" + role)
        if chi is None:
            chi = self.chi_environment
        sp_ = getattr(self, role + "_space")
        if sp_ is None:
            sp_ = self.environment_space
        return dg.BoundaryMPSDiagonal(chi, sp_) if self.diagonal else bm.BoundaryMPS(chi, sp_)


def sample_uniforms(seed: int, index: int, n: int) -> np.ndarray:
    """The uniforms of Born draw ``index`` (1-based) of run ``seed``."""
    return np.random.default_rng([int(seed), int(index)]).random(n)


def same_beta(a, b):
    """``_same_beta`` (``config.jl:63``)."""
    return abs(a - b) <= 64 * EPS * max(1.0, abs(a), abs(b))


def measure_at(c, beta):
    return any(same_beta(b, beta) for b in c.beta_measure)


def temperature_nodes(c):
    """``temperature_nodes`` (``config.jl:68-76``)."""
    nodes = sorted([0.0, c.beta0] + list(c.beta_log) + list(c.beta_measure))
    out = []
    for b in nodes:
        b = c.beta0 if same_beta(b, c.beta0) else b
        if out and same_beta(out[-1], b):
            continue
        out.append(b)
    return out


def step_schedule(start, target, dtau):
    """``_step_schedule`` (``particles.jl:55-64``)."""
    steps = []
    b = float(start)
    while not same_beta(b, target):
        if not target > b:
            raise RuntimeError("evolution requires increasing beta endpoints")
        b = min(target, b + 2 * dtau)
        if same_beta(b, target):
            b = float(target)
        steps.append(b)
    return steps


def observe(state, c, energy):
    """``_observe`` (``particles.jl:35-40``)."""
    if energy:
        return (dg if c.diagonal else sp).measure_energy(state, TFIM(c.J, c.h, c.fields), c.boundary("measurement"),
                                                         record_entropy=c.record_boundary_entropy)
    m = (dg if c.diagonal else bm).lognorm(state, c.boundary("measurement"))
    m.update(energy_total=math.nan, energy_per_site=math.nan, magnetization=math.nan)
    return m


def evolve(state, c, steps, D, space):
    """``_evolve!`` (``particles.jl:66-85``)."""
    maxstate = maxenv = norml = 0.0
    reports = []
    for beta in steps:
        r = fu.evolution_step(state, TFIM(c.J, c.h, c.fields), (beta - state.beta) / 2, D, c.update,
                              c.boundary("environment"), order=c.trotter_order, space=space,
                              record_entropy=c.record_boundary_entropy)
        state.beta = beta
        norml += sum(v for _, v in r["normalizations"])
        maxstate = max(maxstate, r["max_state_truncation"])
        maxenv = max(maxenv, r["max_environment_truncation"])
        reports.append(r)
    return dict(max_state_truncation=maxstate, max_environment_truncation=maxenv, normalization=norml,
                reports=reports)


def run_purification(c: RunConfig):
    """``run_purification`` (``run.jl:2-43``) without file output."""
    state = identity_pepo(c.Lx, c.Ly)
    normalize_state(state)
    rows = []
    for beta in [b for b in temperature_nodes(c) if b <= c.beta0]:
        steps = step_schedule(state.beta, beta, c.delta_tau_pur)
        rep = evolve(state, c, steps, c.D_pur, c.bond_space_pur)
        m = observe(state, c, measure_at(c, beta))
        rows.append(dict(beta=beta, source="purification", energy_total=m["energy_total"],
                         energy_per_site=m["energy_per_site"], lnZ=m["log_norm"],
                         magnetization=m.get("magnetization", math.nan),
                         max_state_truncation=rep["max_state_truncation"],
                         max_environment_truncation=max(rep["max_environment_truncation"],
                                                        m["max_environment_truncation"])))
    return state, rows


def ensemble_statistics(relative, multiplicity, energy, Ns, log_scale=0.0, nsites=1):
    """``ensemble_statistics`` (``ensemble.jl:8-25``)."""
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
    mu2 = np.sum(multiplicity * w ** 2) / Nv
    eta = min(max(mu1 ** 2 / mu2, 1 / Nv), 1.0)

    def sem(f):
        return math.nan if Nv <= 1 else math.sqrt(max(0.0, np.sum(multiplicity * f ** 2) / (Nv * (Nv - 1))))

    measured = bool(np.all(np.isfinite(energy)))
    E = float(np.sum(mass * energy) / total) if measured else math.nan
    Eerr = sem(w * (energy - E) / mu1) if measured else math.nan
    return dict(energy_total=nsites * E, energy_per_site=E, energy_per_site_error=Eerr,
                lnZ=log_scale + pivot + math.log(mu1), lnZ_error=sem((w - mu1) / mu1), eta=eta,
                eta_error=sem((2 * mu1 / mu2) * (w - mu1) - (mu1 ** 2 / mu2 ** 2) * (w ** 2 - mu2)),
                ESS=Nv * eta,
                eta_p=min(max(total ** 2 / (Ns * np.sum(mass ** 2)), 1 / Ns), len(relative) / Ns),
                target_samples=Ns, virtual_samples=Nv, representatives=len(relative))


def run_stochastic(c: RunConfig, checkpoint, uniforms_fn=None):
    """``run_stochastic`` (``run.jl:76-134``) with resampling disabled.

    Returns the curve rows and per-particle records.
    """
    if uniforms_fn is None:
        uniforms_fn = lambda i: sample_uniforms(c.seed, i, c.Lx * c.Ly)
    if c.diagonal:
        cache = dg.DiagonalSamplingCache(checkpoint, c.boundary("sampling"))
        draws = [dg.sample_configuration(cache, uniforms=uniforms_fn(i)) for i in range(1, c.Ns + 1)]
    else:
        cache = sp.SamplingCache(checkpoint, c.boundary("sampling"))
        draws = [sp.sample_configuration(cache, uniforms=uniforms_fn(i)) for i in range(1, c.Ns + 1)]
    grouping = sp.group_configurations([d["configuration"] for d in draws])
    particles = []
    for u, i in enumerate(grouping["first_draw"]):
        d = draws[i]
        state, _ = sp.project_configuration(checkpoint, d["configuration"])
        m = observe(state, c, measure_at(c, c.beta0))
        particles.append(dict(id=i + 1, count=grouping["multiplicity"][u], configuration=d["configuration"],
                              state=state, log_p0=d["log_probability"],
                              relative_log_weight=m["log_norm"] - d["log_probability"],
                              weight_log_scale=0.0, physical_log_norm=m["log_norm"],
                              tensor_log_norm=m["tensor_log_norm"], energy_per_site=m["energy_per_site"],
                              energy_total=m["energy_total"], magnetization=m.get("magnetization", math.nan)))
    nodes = [b for b in temperature_nodes(c) if b >= c.beta0]
    curve = []
    history = []
    for node, beta in enumerate(nodes):
        if node > 0:
            steps = step_schedule(nodes[node - 1], beta, c.delta_tau_peps)
            for p in particles:
                old = p["tensor_log_norm"]
                rep = evolve(p["state"], c, steps, c.D_peps, c.bond_space_peps)
                m = observe(p["state"], c, measure_at(c, beta))
                p["relative_log_weight"] += 2 * rep["normalization"] + (m["tensor_log_norm"] - old)
                p["physical_log_norm"] = m["log_norm"]
                p["tensor_log_norm"] = m["tensor_log_norm"]
                p["energy_total"] = m["energy_total"]
                p["energy_per_site"] = m["energy_per_site"]
                p["magnetization"] = m.get("magnetization", math.nan)
        scale = max(p["weight_log_scale"] for p in particles)
        rel = [p["relative_log_weight"] + (p["weight_log_scale"] - scale) for p in particles]
        st = ensemble_statistics(rel, [p["count"] for p in particles], [p["energy_per_site"] for p in particles],
                                 c.Ns, log_scale=scale, nsites=c.Lx * c.Ly)
        st["beta"] = beta
        curve.append(st)
        history.append([dict(id=p["id"], beta=beta, log_weight=p["weight_log_scale"] + p["relative_log_weight"],
                             energy_per_site=p["energy_per_site"], magnetization=p["magnetization"],
                             count=p["count"]) for p in particles])
    return dict(curve=curve, samples=history, draws=draws, grouping=grouping)
