"""stopeps_b200: the StoPEPS sample-ensemble hot path on one B200.

The public names mirror the reference package StoPEPS.jl v0.2.0
(``src/StoPEPS.jl:32-42``) for the sample-ensemble path: the configuration
types, the row, diagonal and variational boundary methods, the two drivers,
the hot-path functions and the ensemble statistics.
The numerical work runs in ``libstopeps_gpu.so`` (C ABI in
``include/stopeps_gpu.h``).
"""
from .config import (Z2Space, Lattice, TFIM, FullUpdate, BoundaryMPS, BoundaryMPSRow, BoundaryMPSZipUp, BoundaryMPSDiagonal, BoundaryMPSRowVariational, BoundaryMPSDiagonalVariational, ResamplingOptions,
                     SymmetryBasis, RunConfig, validate_config, temperature_nodes, parameter_dict)
from .engine import (Engine, DeviceState, SamplingCache, normalize_state, evolution_step, lognorm, lognorm_gradient, lognorm_field_gradient,
                     measure_energy, sample_configuration, sample_batch, project_configuration,
                     project_batch, evolution_step_batch, measure_energy_batch, lognorm_batch,
                     sample_conditionals, sample_probability_batch)
from .driver import (run_purification, run_stochastic, ensemble_statistics, group_configurations,
                     sample_uniforms, step_schedule, ThermalCheckpoint, Particle, RESULT_SCHEMA_VERSION)
from .autodiff import LognormFunction, lognorm_differentiable
from . import _lib
from .build import build, LIB as LIBRARY_PATH
from .parallel import SerialExecution, TorchExecution
from .checkpoint import save_checkpoint, load_checkpoint, CHECKPOINT_FORMAT
from .models import physical_space, dense_hamiltonian, exact_thermal_observables, identity_pepo, validate_state
from .results import save_result, load_result, save_run_result
from . import results as Results
from . import synthetic
from . import bench_states

__all__ = [
    "Z2Space", "Lattice", "TFIM", "FullUpdate", "BoundaryMPS", "BoundaryMPSRow", "ResamplingOptions",
    "SymmetryBasis", "RunConfig", "validate_config", "temperature_nodes", "parameter_dict", "Engine",
    "DeviceState", "SamplingCache", "normalize_state", "evolution_step", "lognorm", "lognorm_gradient", "lognorm_field_gradient", "LognormFunction", "lognorm_differentiable", "measure_energy",
    "sample_configuration", "sample_batch", "project_configuration", "project_batch", "evolution_step_batch",
    "measure_energy_batch", "lognorm_batch", "sample_conditionals", "sample_probability_batch",
    "run_purification", "run_stochastic",
    "ensemble_statistics", "group_configurations", "sample_uniforms", "step_schedule", "ThermalCheckpoint",
    "Particle", "RESULT_SCHEMA_VERSION", "build", "LIBRARY_PATH", "save_checkpoint", "load_checkpoint",
    "CHECKPOINT_FORMAT", "physical_space", "dense_hamiltonian", "exact_thermal_observables", "identity_pepo",
    "validate_state", "save_result", "load_result", "save_run_result", "Results",
]
