"""Host logic of the engine package (no GPU): configuration, schedules,
statistics and the C-ABI library's exported symbols."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

from oracle import driver as odr

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_validate_config_defaults_and_errors(sps):
    c = sps.RunConfig()
    assert sps.validate_config(c) is c
    assert c.chi_sampling == c.chi_environment == c.chi_measurement == 32
    with pytest.raises(ValueError):
        sps.validate_config(sps.RunConfig(delta_tau_pur=0.0))
    with pytest.raises(ValueError):
        sps.validate_config(sps.RunConfig(Ns=1))          # resampling needs Ns >= 2
    with pytest.raises(ValueError):
        sps.validate_config(sps.RunConfig(trotter_order=3))
    with pytest.raises(ValueError):
        sps.TFIM(physical_space=sps.Z2Space(2, 2))


def test_temperature_nodes_and_schedule_match_oracle(sps):
    c = sps.RunConfig(beta0=0.5, beta_log=[1.0, 2.0, 3.0, 4.0], beta_measure=[0.5, 1.0, 2.0, 3.0, 4.0])
    oc = odr.RunConfig(beta0=0.5, beta_log=[1.0, 2.0, 3.0, 4.0], beta_measure=[0.5, 1.0, 2.0, 3.0, 4.0])
    assert sps.temperature_nodes(c) == odr.temperature_nodes(oc) == [0.0, 0.5, 1.0, 2.0, 3.0, 4.0]
    s = sps.step_schedule(0.5, 1.0, 0.05)
    assert s == odr.step_schedule(0.5, 1.0, 0.05)
    assert len(s) == 5 and s[-1] == 1.0
    assert sps.step_schedule(0.0, 0.07, 0.025) == [0.05, 0.07]
    with pytest.raises(ValueError):
        sps.step_schedule(1.0, 0.5, 0.05)


def test_ensemble_statistics_matches_oracle(sps):
    rng = np.random.default_rng(0)
    rel = rng.normal(size=9)
    mult = rng.integers(1, 4, size=9)
    en = rng.normal(size=9)
    a = sps.ensemble_statistics(rel, mult, en, 12, log_scale=0.3, nsites=16)
    b = odr.ensemble_statistics(rel, mult, en, 12, log_scale=0.3, nsites=16)
    for k in b:
        assert (math.isnan(a[k]) and math.isnan(b[k])) or abs(a[k] - b[k]) < 1e-14, k
    with pytest.raises(ValueError):
        sps.ensemble_statistics([], [], [], 1)
    with pytest.raises(ValueError):
        sps.ensemble_statistics([np.inf], [1], [0.0], 1)


def test_group_configurations(sps):
    cfgs = [np.array([[1, 2], [1, 1]]), np.array([[1, 1], [1, 1]]), np.array([[1, 2], [1, 1]])]
    g = sps.group_configurations(cfgs)
    assert g == dict(first_draw=[1, 2], multiplicity=[2, 1], draw_to_group=[1, 2, 1])


def test_sample_uniforms_are_reproducible(sps):
    a = sps.sample_uniforms(7, 3, 16)
    assert np.array_equal(a, sps.sample_uniforms(7, 3, 16))
    assert np.array_equal(a, odr.sample_uniforms(7, 3, 16))
    assert not np.array_equal(a, sps.sample_uniforms(7, 4, 16))
    with pytest.raises(ValueError):
        sps.sample_uniforms(-1, 1, 4)


def test_library_exports_every_declared_symbol(sps):
    header = open(os.path.join(ROOT, "include", "stopeps_gpu.h")).read()
    declared = set(re.findall(r"\b(sps_[a-z_0-9]+)\s*\(", header))
    lib = ctypes.CDLL(sps.LIBRARY_PATH)
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    assert declared >= set(sps._lib.EXPORTS)


def test_create_without_device_fails_loudly(sps):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(sps._lib.EngineError):
        sps.Engine(2, 2)


def test_stored_benchmark_state_layout(sps):
    """The stored purified 8x8 PEPO: 64 sites, legs (W,N,Pout,Paux,E,S) with the
    D = 6 (3+3) bulk bonds, trivial outer legs, sector-sorted blocks whose
    parity-odd entries are zero."""
    import numpy as np
    sites, dims, beta, log_amplitude = sps.bench_states.load()
    assert len(sites) == 64 and dims.shape == (64, 6, 2)
    assert abs(beta - 0.4) < 1e-14 and np.isfinite(log_amplitude)
    for i, (a, d) in enumerate(zip(sites, dims)):
        x, y = i % 8, i // 8
        assert tuple(d[2]) == (1, 1) and tuple(d[3]) == (1, 1)
        assert tuple(d[0]) == ((1, 0) if x == 0 else (3, 3))
        assert tuple(d[5]) == ((1, 0) if y == 7 else (3, 3))
        par = np.zeros(a.shape, np.int64)
        for k, (n0, n1) in enumerate(d):
            p = np.concatenate([np.zeros(n0, np.int64), np.ones(n1, np.int64)])
            sh = [1] * 6
            sh[k] = n0 + n1
            par = par + p.reshape(sh)
        assert np.all(a[par % 2 == 1] == 0.0)
        assert np.linalg.norm(a) > 0


@pytest.mark.parametrize("Lx,Ly", [(1, 1), (1, 4), (4, 1), (3, 2), (4, 5)])
def test_diagonal_draw_order_matches_oracle(sps, Lx, Ly):
    """``_diagonal_order``: the host's order (used for the parameter record and
    the uniforms of a diagonal draw) is the oracle's, a permutation of the sites."""
    from oracle import diagonal as dg
    order = sps.config.diagonal_order(Lx, Ly)
    assert order == dg.draw_order(Lx, Ly)
    assert sorted(order) == sorted((x, y) for x in range(Lx) for y in range(Ly))


def test_boundary_methods_and_parameter_records(sps):
    """The boundary methods a RunConfig may name, their records
    (``config.jl:129-136``) and their option checks."""
    names = {sps.BoundaryMPS: ("BoundaryMPS-Row", "row_major"),
             sps.BoundaryMPSDiagonal: ("BoundaryMPS-Diagonal",
                                       "x+y_ascending; even_diagonal_x_ascending; odd_diagonal_x_descending"),
             sps.BoundaryMPSRowVariational: ("BoundaryMPS-Row-Variational", "row_major"),
             sps.BoundaryMPSDiagonalVariational: ("BoundaryMPS-Diagonal-Variational",
                                                  "x+y_ascending; even_diagonal_x_ascending; "
                                                  "odd_diagonal_x_descending")}
    for cls, (name, order) in names.items():
        c = sps.RunConfig(lattice=sps.Lattice(3, 2), contraction=cls)
        sps.validate_config(c)
        p = sps.parameter_dict(c)
        assert p["contraction"] == name and p["contraction_order"] == order
        assert isinstance(c.boundary("sampling"), cls)
    with pytest.raises(ValueError):
        sps.validate_config(sps.RunConfig(contraction=sps.BoundaryMPSZipUp))
    for cls in (sps.BoundaryMPSRowVariational, sps.BoundaryMPSDiagonalVariational):
        for bad in (dict(chi=0), dict(chi=4, max_sweep=0), dict(chi=4, threshold_sweep=float("nan"))):
            with pytest.raises(ValueError):
                cls(**bad)
    with pytest.raises(ValueError):
        sps.BoundaryMPSDiagonalVariational(4, target_cache_bytes=-1)
