"""The oracle's row variational boundary MPS (``src/contraction/row_variational.jl``)
pinned on the CPU.

At a chi above every bond the variational fit reproduces the exact row
contraction (lnZ, energy, Born probabilities); at a truncating chi its fit is
at least as good as the compression's in lnZ; sweeps stop on the
``threshold_sweep`` rule, run the whole budget with a zero threshold, and
one-column lattices take the direct projection.
"""
import itertools
import math

import numpy as np
import pytest

from oracle import boundary as bm, driver as dr, model as md, sampling as sp, variational as va


def _state(Lx, Ly, h=1.0, D=3, beta=0.3):
    c = dr.RunConfig(Lx=Lx, Ly=Ly, J=1.0, h=h, beta0=beta, beta_log=[beta], beta_measure=[beta],
                     delta_tau_pur=0.05, D_pur=D, D_peps=D, chi_environment=64, Ns=1)
    return dr.run_purification(c)[0]


def test_exact_chi_equals_exact_contraction():
    st = _state(3, 2, h=0.9)
    m = md.TFIM(1.0, 0.9)
    a = sp.measure_energy(st, m, bm.BoundaryMPS(200))
    b = sp.measure_energy(st, m, va.BoundaryMPSRowVariational(200))
    for k in ("energy_total", "log_norm", "x_sum", "zz_sum"):
        assert abs(a[k] - b[k]) <= 1e-12 * max(1.0, abs(a[k])), k
    ca, cb = sp.SamplingCache(st, bm.BoundaryMPS(200)), sp.SamplingCache(st, va.BoundaryMPSRowVariational(200))
    total = 0.0
    for bits in itertools.product([1, 2], repeat=6):
        cfg = [[bits[x + 3 * y] for y in range(2)] for x in range(3)]
        p = sp.sample_configuration(ca, configuration=cfg)["log_probability"]
        q = sp.sample_configuration(cb, configuration=cfg)["log_probability"]
        assert abs(p - q) < 1e-11
        total += math.exp(q)
    assert abs(total - 1.0) < 1e-12


def test_truncated_fit_and_sweep_records():
    st = _state(4, 3)
    exact = bm.lognorm(st, bm.BoundaryMPS(400))["log_norm"]
    for chi in (4, 8):
        row = bm.lognorm(st, bm.BoundaryMPS(chi))
        var = bm.lognorm(st, va.BoundaryMPSRowVariational(chi))
        assert abs(var["log_norm"] - exact) <= 1.5 * abs(row["log_norm"] - exact) + 1e-13
        assert var["max_environment_truncation"] > 0
        s = var["boundary_variational"]
        assert len(s["layers"]) == 3 and s["fallback_count"] == 0
        assert all(r["stop_reason"] in ("threshold_sweep", "sweep_limit") for r in s["layers"])
    full = bm.lognorm(st, va.BoundaryMPSRowVariational(8, threshold_sweep=0.0, max_sweep=3))
    assert [r["sweeps"] for r in full["boundary_variational"]["layers"]] == [3, 3, 3]
    assert full["boundary_variational"]["sweep_limit_hits"] == 3
    assert abs(full["log_norm"] - exact) < 1e-9
    e = sp.measure_energy(st, md.TFIM(1.0, 1.0), va.BoundaryMPSRowVariational(16), record_entropy=True)
    ref = sp.measure_energy(st, md.TFIM(1.0, 1.0), bm.BoundaryMPS(64))
    assert abs(e["energy_per_site"] - ref["energy_per_site"]) < 1e-10
    assert np.all(np.isfinite(e["Se"]["north"])) and np.nanmax(e["Se"]["north"]) > 0


def test_one_column_takes_the_direct_projection():
    st = _state(1, 3, D=2)
    a = bm.lognorm(st, bm.BoundaryMPS(16))
    b = bm.lognorm(st, va.BoundaryMPSRowVariational(16))
    assert abs(a["log_norm"] - b["log_norm"]) < 1e-12
    assert all(r["stop_reason"] == "direct" for r in b["boundary_variational"]["layers"])


def test_space_map_and_options():
    P, Q = np.array([0, 0, 0, 1], np.int8), np.array([0, 1, 1], np.int8)
    M = va.space_map(P, Q)
    assert M.shape == (3, 4)
    np.testing.assert_array_equal(M, [[1, 0, 0, 0], [0, 0, 0, 1], [0, 0, 0, 0]])
    v = va.identity_vector(np.zeros(9, np.int8))
    assert abs(np.linalg.norm(v.a) - 1) < 1e-15 and np.count_nonzero(v.a) == 3
    for bad in (dict(chi=0), dict(chi=4, max_sweep=0), dict(chi=4, threshold_sweep=-1.0)):
        with pytest.raises(ValueError):
            va.BoundaryMPSRowVariational(**bad)


def test_diagonal_variational_exact_and_truncated():
    """``diagonal_variational.jl``: exact at a chi above every bond (energy and
    every Born probability equal the row contraction's), as accurate as the
    diagonal SVD absorption at a truncating chi, records per layer, the whole
    sweep budget with a zero threshold, and the full update runs on it."""
    from oracle import diagonal as dg, diagonal_variational as dv, full_update as fu
    st = _state(3, 2, h=0.9)
    m = md.TFIM(1.0, 0.9)
    a = sp.measure_energy(st, m, bm.BoundaryMPS(200))
    b = dg.measure_energy(st, m, dv.BoundaryMPSDiagonalVariational(200))
    for k in ("energy_total", "log_norm", "x_sum", "zz_sum"):
        assert abs(a[k] - b[k]) <= 1e-12 * max(1.0, abs(a[k])), k
    ca = sp.SamplingCache(st, bm.BoundaryMPS(200))
    cb = dg.DiagonalSamplingCache(st, dv.BoundaryMPSDiagonalVariational(200))
    for bits in itertools.product([1, 2], repeat=6):
        cfg = [[bits[x + 3 * y] for y in range(2)] for x in range(3)]
        assert abs(sp.sample_configuration(ca, configuration=cfg)["log_probability"]
                   - dg.sample_configuration(cb, configuration=cfg)["log_probability"]) < 1e-11
    st = _state(4, 3)
    exact = bm.lognorm(st, bm.BoundaryMPS(400))["log_norm"]
    for chi in (4, 8):
        svd = dg.lognorm(st, dg.BoundaryMPSDiagonal(chi))
        var = dg.lognorm(st, dv.BoundaryMPSDiagonalVariational(chi))
        assert abs(var["log_norm"] - exact) <= 1.5 * abs(svd["log_norm"] - exact) + 1e-13
        layers = var["boundary_variational"]["layers"]
        assert len(layers) == dg.layer_count(4, 3) and var["boundary_variational"]["fallback_count"] == 0
        assert {r["stop_reason"] for r in layers} <= {"direct", "threshold_sweep", "sweep_limit"}
    full = dg.lognorm(st, dv.BoundaryMPSDiagonalVariational(8, threshold_sweep=0.0, max_sweep=2))
    assert all(r["sweeps"] == 2 for r in full["boundary_variational"]["layers"] if r["stop_reason"] != "direct")
    out = []
    for method in (bm.BoundaryMPS(400), dv.BoundaryMPSDiagonalVariational(400)):
        s = md.identity_pepo(3, 2)
        md.normalize_state(s)
        fu.evolution_step(s, m, 0.05, 4, fu.FullUpdate(), method)
        out.append(sp.measure_energy(s, m, bm.BoundaryMPS(400))["energy_per_site"])
    assert abs(out[0] - out[1]) < 1e-12
    with pytest.raises(ValueError):
        dv.BoundaryMPSDiagonalVariational(4, None, target_cache_bytes=-1)
