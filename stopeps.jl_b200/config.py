"""Run configuration, mirroring the reference's ``RunConfig`` and friends.

``RunConfig`` (``src/driver/config.jl:28-62``), ``ResamplingOptions``
(``config.jl:10-18``), ``FullUpdate`` (``src/evolution/full_update.jl:11-17``),
``BoundaryMPS`` (``src/contraction/boundary_mps.jl:11-18``), ``TFIM``
(``src/models/tfim.jl:9-19``) and ``Lattice`` (``src/states/finite.jl:1-9``)
keep their field names and defaults.  Z2 spaces are written
``Z2Space(n0, n1)`` (even and odd multiplicities).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, fields
from typing import Optional

EPS = 2.220446049250313e-16


@dataclass(frozen=True)
class Z2Space:
    """``Z2Space(0=>n0, 1=>n1)``."""
    n0: int
    n1: int

    @property
    def dim(self):
        return self.n0 + self.n1

    def as_tuple(self):
        return (self.n0, self.n1)


@dataclass(frozen=True)
class Lattice:
    Lx: int
    Ly: int

    def __post_init__(self):
        if not (self.Lx > 0 and self.Ly > 0):
            raise ValueError("lattice dimensions must be positive")

    def __len__(self):
        return self.Lx * self.Ly


@dataclass(frozen=True)
class TFIM:
    """H = -J sum ZZ - h sum X, Z2-symmetric physical space (X eigenbasis).

    ``fields`` (optional, Lx*Ly values in x + y*Lx order) replaces the uniform
    h by a transverse field per site, H = -J sum ZZ - sum_i h_i X_i: an
    extension of the reference's model (one h) for per-site lnZ gradients
    (d lnZ / d h_i = beta <X_i>).  ``None`` is the reference's model."""
    J: float = 1.0
    h: float = 0.7
    physical_space: Z2Space = Z2Space(1, 1)
    fields: Optional[tuple] = None

    def __post_init__(self):
        if self.physical_space != Z2Space(1, 1):
            raise ValueError("TFIM supports Z2Space(0=>1,1=>1) in the X eigenbasis")
        if self.fields is not None:
            f = tuple(float(v) for v in self.fields)
            if not f or not all(math.isfinite(v) for v in f):
                raise ValueError("per-site fields must be a nonempty sequence of finite numbers")
            object.__setattr__(self, "fields", f)

    def field(self, x, y, Lx):
        """The transverse field at 0-based site (x, y)."""
        return self.h if self.fields is None else self.fields[x + y * Lx]


@dataclass(frozen=True)
class FullUpdate:
    max_iterations: int = 4
    error_tolerance: float = 1e-8
    diagonal_shift: float = 1e-10
    linear_max_iterations: int = 24
    linear_tolerance: float = 1e-9


@dataclass(frozen=True)
class BoundaryMPS:
    chi: int = 32
    sector_space: Optional[Z2Space] = None


BoundaryMPSRow = BoundaryMPS


@dataclass(frozen=True)
class BoundaryMPSZipUp(BoundaryMPS):
    """Row boundary MPS whose rows are absorbed by one zip-up sweep of
    truncated SVDs (no canonical form), this library's variant of
    ``BoundaryMPS``; same ``chi`` and ``sector_space`` truncation
    (``boundary_mps.jl:18``)."""


@dataclass(frozen=True)
class BoundaryMPSDiagonal(BoundaryMPS):
    """``BoundaryMPSDiagonal(chi, sector_space)`` (``src/contraction/diagonal_mps.jl:3-9``):
    anti-diagonal layers x + y = t absorbed as site blocks, with the same ``chi``
    and sector budget.  Taken by ``lognorm``, ``measure_energy``,
    ``SamplingCache`` and the full update's bond environments
    (``src/evolution/diagonal_update.jl``); ``RunConfig(contraction=...)``."""


@dataclass(frozen=True)
class BoundaryMPSDiagonalVariational(BoundaryMPSDiagonal):
    """``BoundaryMPSDiagonalVariational(chi; sector_space, max_sweep=4, threshold_sweep=1e-8,
    target_cache_bytes)`` (``src/contraction/diagonal_variational.jl:12-30``): every
    diagonal layer absorbed by a two-site variational fit; the engine keeps no
    target-block cache, so ``target_cache_bytes`` is only validated."""
    max_sweep: int = 4
    threshold_sweep: float = 1e-8
    target_cache_bytes: int = 256 * 1024 ** 2

    def __post_init__(self):
        if self.chi < 1:
            raise ValueError("chi must be positive")
        if self.max_sweep < 1:
            raise ValueError("max_sweep must be positive")
        if not (math.isfinite(self.threshold_sweep) and self.threshold_sweep >= 0):
            raise ValueError("threshold_sweep must be finite and nonnegative")
        if self.target_cache_bytes < 0:
            raise ValueError("target_cache_bytes must be nonnegative")


@dataclass(frozen=True)
class BoundaryMPSRowVariational(BoundaryMPS):
    """``BoundaryMPSRowVariational(chi; sector_space, max_sweep=4, threshold_sweep=1e-8)``
    (``src/contraction/row_variational.jl:10-25``): every row absorbed by a
    two-site variational fit instead of the exact compression; sweeps stop at
    ``max_sweep`` or when the squared norm changes by at most ``threshold_sweep``."""
    max_sweep: int = 4
    threshold_sweep: float = 1e-8

    def __post_init__(self):
        if self.chi < 1:
            raise ValueError("chi must be positive")
        if self.max_sweep < 1:
            raise ValueError("max_sweep must be positive")
        if not (math.isfinite(self.threshold_sweep) and self.threshold_sweep >= 0):
            raise ValueError("threshold_sweep must be finite and nonnegative")


@dataclass(frozen=True)
class ResamplingOptions:
    enabled: bool = True
    eta_th: float = 0.7
    lambda_max: float = 0.999
    lambda_tolerance: float = 1e-8
    lambda_threshold: float = 0.2
    max_resample_sweep: int = 3
    score_batch_size: int = 32


class SymmetryBasis:
    """Sample the abelian charge states of the auxiliary leg (``src/sampling/basis.jl:19``)."""

    def __eq__(self, other):
        return isinstance(other, SymmetryBasis)

    def __repr__(self):
        return "SymmetryBasis()"


@dataclass
class RunConfig:
    lattice: Lattice = Lattice(2, 2)
    model: TFIM = TFIM()
    beta0: float = 0.1
    beta_log: list = field(default_factory=lambda: [round(0.05 * k, 10) for k in range(7)])
    beta_measure: list = field(default_factory=lambda: [0.0, 0.1, 0.2, 0.3])
    delta_tau_pur: float = 0.025
    delta_tau_peps: float = 0.025
    D_pur: int = 4
    D_peps: int = 4
    bond_space_pur: Optional[Z2Space] = None
    bond_space_peps: Optional[Z2Space] = None
    chi_environment: int = 32
    chi_sampling: Optional[int] = None
    chi_measurement: Optional[int] = None
    chi_proposal: Optional[int] = None
    environment_space: Optional[Z2Space] = None
    sampling_space: Optional[Z2Space] = None
    measurement_space: Optional[Z2Space] = None
    proposal_space: Optional[Z2Space] = None
    sampling_basis: object = field(default_factory=SymmetryBasis)
    trotter_order: int = 2
    update: FullUpdate = FullUpdate()
    contraction: type = BoundaryMPS
    record_boundary_entropy: bool = True
    Ns: int = 16
    seed: int = 20260924
    resampling: ResamplingOptions = ResamplingOptions()
    save_interval_seconds: float = 3600.0
    output_directory: Optional[str] = None
    overwrite_output: bool = False

    def __post_init__(self):
        # keyword defaults that follow other fields (config.jl:41-47)
        if self.chi_sampling is None:
            self.chi_sampling = self.chi_environment
        if self.chi_measurement is None:
            self.chi_measurement = self.chi_environment
        if self.chi_proposal is None:
            self.chi_proposal = self.chi_sampling
        if self.sampling_space is None:
            self.sampling_space = self.environment_space
        if self.measurement_space is None:
            self.measurement_space = self.environment_space
        if self.proposal_space is None:
            self.proposal_space = self.sampling_space

    def boundary(self, role: str) -> BoundaryMPS:
        """``_boundary(c, role)`` (``src/driver/particles.jl:27-34``)."""
        return self.contraction(getattr(self, "chi_" + role), getattr(self, role + "_space"))


def same_beta(a, b):
    """``_same_beta`` (``config.jl:63``)."""
    return abs(a - b) <= 64 * EPS * max(1.0, abs(a), abs(b))


def measure_at(c: RunConfig, beta):
    return any(same_beta(b, beta) for b in c.beta_measure)


def temperature_nodes(c: RunConfig):
    """Sorted output grid from beta_log, beta_measure, 0 and beta0 (``config.jl:68-76``)."""
    nodes = sorted([0.0, c.beta0] + list(c.beta_log) + list(c.beta_measure))
    out = []
    for b in nodes:
        b = c.beta0 if same_beta(b, c.beta0) else b
        if out and same_beta(out[-1], b):
            continue
        out.append(float(b))
    return out


def validate_config(c: RunConfig) -> RunConfig:
    """``validate_config`` (``config.jl:80-114``) for the row boundary-MPS path."""
    if c.contraction not in (BoundaryMPS, BoundaryMPSDiagonal, BoundaryMPSRowVariational,
                             BoundaryMPSDiagonalVariational):
        raise ValueError("this engine implements the row, diagonal and variational boundary-MPS contractions "
                         "(BoundaryMPS/BoundaryMPSRow, BoundaryMPSDiagonal, BoundaryMPSRowVariational, "
                         "BoundaryMPSDiagonalVariational)")
    grid = [c.beta0] + list(c.beta_log) + list(c.beta_measure)
    if not all(math.isfinite(b) and b >= 0 for b in grid):
        raise ValueError("invalid beta grid")
    if not all(math.isfinite(x) and x > 0 for x in (c.delta_tau_pur, c.delta_tau_peps)):
        raise ValueError("delta_tau must be positive")
    if min(c.D_pur, c.D_peps, c.chi_environment, c.chi_sampling, c.chi_measurement, c.chi_proposal, c.Ns) < 1:
        raise ValueError("dimensions and sample count must be positive")
    if not (c.seed >= 0 and c.trotter_order in (1, 2)):
        raise ValueError("invalid seed or Trotter order")
    if not (math.isfinite(c.save_interval_seconds) and c.save_interval_seconds >= 0):
        raise ValueError("invalid save interval")
    r = c.resampling
    if not (0 <= r.eta_th <= 1 and 0 <= r.lambda_max < 1 and r.lambda_tolerance > 0
            and math.isfinite(r.lambda_threshold) and 0 <= r.lambda_threshold < 1
            and r.max_resample_sweep >= 1 and r.score_batch_size > 0):
        raise ValueError("invalid resampling options")
    if r.enabled and c.Ns < 2:
        raise ValueError("resampling needs Ns >= 2")
    u = c.update
    if not (u.max_iterations >= 0 and u.linear_max_iterations > 0
            and all(math.isfinite(x) and x >= 0 for x in (u.error_tolerance, u.diagonal_shift, u.linear_tolerance))):
        raise ValueError("invalid full-update options")
    if not (math.isfinite(c.model.J) and math.isfinite(c.model.h)):
        raise ValueError("nonfinite model parameter")
    if c.model.fields is not None and len(c.model.fields) != c.lattice.Lx * c.lattice.Ly:
        raise ValueError("per-site fields need one value per lattice site")
    for V in (c.bond_space_pur, c.bond_space_peps, c.environment_space, c.sampling_space,
              c.measurement_space, c.proposal_space):
        if V is None:
            continue
        if not (isinstance(V, Z2Space) and V.dim > 0 and V.n0 >= 0 and V.n1 >= 0):
            raise ValueError("sector budgets must be nondual, nonempty spaces with the model symmetry")
    if not isinstance(c.sampling_basis, SymmetryBasis):
        raise ValueError("symmetric sampling requires SymmetryBasis()")
    return c


def diagonal_order(Lx, Ly):
    """``_diagonal_order`` (``src/contraction/diagonal_mps.jl:111``): the 0-based sites
    (x, y) by anti-diagonals x + y = 0, 1, ..., even ones by increasing x, odd
    ones by decreasing x; the order in which a diagonal draw visits them."""
    out = []
    for t in range(Lx + Ly - 1):
        layer = [(x, t - x) for x in range(max(0, t - Ly + 1), min(Lx - 1, t) + 1)]
        out.extend(reversed(layer) if t % 2 else layer)
    return out


def parameter_dict(c: RunConfig) -> dict:
    """Plain-container encoding of the configuration (``config.jl:117-185``, subset)."""
    def enc(x):
        if isinstance(x, (int, float, str, bool)) or x is None:
            return x
        if isinstance(x, (list, tuple)):
            return [enc(v) for v in x]
        if isinstance(x, type):
            return x.__name__
        if isinstance(x, Z2Space):
            return {"sector_type": "Z2Irrep", "dual": False,
                    "sectors": [{"sector": "0", "multiplicity": x.n0}, {"sector": "1", "multiplicity": x.n1}]}
        if hasattr(x, "__dataclass_fields__"):
            d = {"type": type(x).__name__}
            d.update({f.name: enc(getattr(x, f.name)) for f in fields(x)
                      if not (isinstance(x, TFIM) and f.name == "fields" and x.fields is None)})
            return d
        return repr(x)
    d = {f.name: enc(getattr(c, f.name)) for f in fields(c)}
    diagonal = issubclass(c.contraction, BoundaryMPSDiagonal)
    d["contraction"] = {BoundaryMPSDiagonal: "BoundaryMPS-Diagonal",
                        BoundaryMPSDiagonalVariational: "BoundaryMPS-Diagonal-Variational",
                        BoundaryMPSRowVariational: "BoundaryMPS-Row-Variational"}.get(c.contraction, "BoundaryMPS-Row")
    d["sampling_site_order"] = (
        [(x + 1, y + 1) for x, y in diagonal_order(c.lattice.Lx, c.lattice.Ly)] if diagonal
        else [(x + 1, y + 1) for y in range(c.lattice.Ly) for x in range(c.lattice.Lx)])
    d["contraction_order"] = ("x+y_ascending; even_diagonal_x_ascending; odd_diagonal_x_descending" if diagonal
                              else "row_major")
    d["state_truncation_metric"] = "relative_squared_FU_residual"
    d["full_update_algorithm"] = "environment_gauge_SVD_ALS"
    d["full_update_algorithm_revision"] = 2
    d["environment_truncation_metric"] = "canonical_SVD_relative_discarded_weight"
    d["boundary_entropy_convention"] = "pretruncation_Schmidt_entropy; nats; sector_dimension_weighted"
    d["uncertainty"] = "conditional_particle_delta_method; shared_history_scale_fixed"
    d["rng_algorithm"] = "explicit_uniforms (numpy default_rng([seed, index]))"
    d["factor_time_convention"] = "tau=beta/2"
    d["temperature_nodes"] = temperature_nodes(c)
    return d
