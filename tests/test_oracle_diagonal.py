"""The oracle's diagonal boundary MPS (``src/contraction/diagonal_mps.jl``,
``src/sampling/diagonal_born.jl``, ``src/measurement/diagonal_energy.jl``),
pinned on the CPU.

With chi above every bond the diagonal contraction is exact, so lnZ, the
energy, the per-site <X> and every configuration's Born probability must
equal the exact row contraction (itself pinned to exact diagonalisation) to
rounding; the Born distribution sums to one; truncating chi converges to the
exact value; and lattices with one row or column go through the same code.
"""
import itertools
import math

import numpy as np
import pytest

from oracle import boundary as bm, diagonal as dg, driver as dr, model as md, sampling as sp

EXACT = 1e-12


def _state(Lx, Ly, h=0.9, D=2, beta=0.2, fields=None):
    c = dr.RunConfig(Lx=Lx, Ly=Ly, J=1.0, h=h, beta0=beta, beta_log=[beta], beta_measure=[beta],
                     delta_tau_pur=0.05, D_pur=D, D_peps=D, chi_environment=64, Ns=1, fields=fields)
    return dr.run_purification(c)[0]


def _configs(Lx, Ly):
    for bits in itertools.product([1, 2], repeat=Lx * Ly):
        yield [[bits[x + Lx * y] for y in range(Ly)] for x in range(Lx)]


@pytest.mark.parametrize("Lx,Ly", [(1, 1), (1, 3), (3, 1), (2, 2), (3, 2)])
def test_exact_chi_equals_row_contraction(Lx, Ly):
    st = _state(Lx, Ly, D=3 if Lx * Ly == 6 else 2)
    m = md.TFIM(1.0, 0.9)
    a = sp.measure_energy(st, m, bm.BoundaryMPS(200))
    b = dg.measure_energy(st, m, dg.BoundaryMPSDiagonal(200))
    for k in ("energy_total", "log_norm", "tensor_log_norm", "x_sum", "zz_sum"):
        assert abs(a[k] - b[k]) <= EXACT * max(1.0, abs(a[k])), k
    np.testing.assert_allclose(b["site_x"], a["site_x"], atol=EXACT)
    assert abs(dg.lognorm(st, dg.BoundaryMPSDiagonal(200))["log_norm"] - a["log_norm"]) <= EXACT * abs(a["log_norm"])
    ca, cb = sp.SamplingCache(st, bm.BoundaryMPS(200)), dg.DiagonalSamplingCache(st, dg.BoundaryMPSDiagonal(200))
    total = 0.0
    for cfg in _configs(Lx, Ly):
        p = sp.sample_configuration(ca, configuration=cfg)["log_probability"]
        q = dg.sample_configuration(cb, configuration=cfg)
        assert abs(p - q["log_probability"]) < 1e-12
        assert len(q["conditionals"]) == Lx * Ly
        total += math.exp(q["log_probability"])
    assert abs(total - 1.0) < 1e-12


def test_physical_kind_equals_row_contraction():
    """The resampling proposal over a projected PEPS: the same distribution as
    the row method's at exact chi, zero mass off the PEPS's total charge."""
    st = _state(3, 2, D=3)
    peps, _ = sp.project_configuration(st, [[1, 2], [2, 1], [1, 1]])
    ca = sp.SamplingCache(peps, bm.BoundaryMPS(200), kind="physical")
    cb = dg.DiagonalSamplingCache(peps, dg.BoundaryMPSDiagonal(200), kind="physical")
    total = 0.0
    for cfg in _configs(3, 2):
        p = sp.sample_configuration(ca, configuration=cfg)["log_probability"]
        q = dg.sample_configuration(cb, configuration=cfg)
        if p == -math.inf:
            assert q["log_probability"] == -math.inf
            continue
        assert abs(p - q["log_probability"]) < 1e-12
        assert len([r for r in q["repairs"] if "reason" not in r]) == 6
        total += math.exp(q["log_probability"])
    assert abs(total - 1.0) < 1e-12
    with pytest.raises(ValueError):
        dg.DiagonalSamplingCache(st, dg.BoundaryMPSDiagonal(8), kind="physical")


def test_draws_follow_uniforms_and_the_draw_order():
    """A draw consumes its uniforms in the anti-diagonal order (even layers by
    increasing x, odd layers by decreasing x) and evaluating the drawn
    configuration returns the same log probability and conditionals."""
    assert dg.draw_order(3, 2) == [(0, 0), (1, 0), (0, 1), (1, 1), (2, 0), (2, 1)]
    st = _state(3, 2, D=3)
    cache = dg.DiagonalSamplingCache(st, dg.BoundaryMPSDiagonal(6))
    u = np.random.default_rng(5).random(6)
    r = dg.sample_configuration(cache, uniforms=u)
    again = dg.sample_configuration(cache, configuration=r["configuration"])
    assert again["log_probability"] == r["log_probability"]
    assert again["conditionals"] == r["conditionals"]
    # the first site drawn is (0,0) with uniform u[0]
    p0 = r["conditionals"][0]
    first = r["configuration"][0][0]
    if first == 1:
        assert u[0] < p0
    else:
        assert u[0] >= 1 - p0


def test_truncation_converges_to_exact():
    st = _state(4, 3, h=1.0, D=3, beta=0.3)
    exact = bm.lognorm(st, bm.BoundaryMPS(400))["log_norm"]
    errs = []
    for chi in (4, 8, 16):
        r = dg.lognorm(st, dg.BoundaryMPSDiagonal(chi))
        errs.append(abs(r["log_norm"] - exact))
        assert r["max_environment_truncation"] >= 0
    assert errs[2] < 1e-10 and errs[0] > errs[2]
    e = dg.measure_energy(st, md.TFIM(1.0, 1.0), dg.BoundaryMPSDiagonal(16), record_entropy=True)
    ref = sp.measure_energy(st, md.TFIM(1.0, 1.0), bm.BoundaryMPS(64))
    assert abs(e["energy_per_site"] - ref["energy_per_site"]) < 1e-10
    assert e["max_boundary_entropy"] > 0
    assert np.nanmax(e["Se"]["northwest"]) == pytest.approx(e["max_boundary_entropy"]) or \
        np.nanmax(e["Se"]["southeast"]) == pytest.approx(e["max_boundary_entropy"])


def test_sector_budget_and_fields():
    """A sector budget caps each parity block of the opened bonds; per-site
    fields enter the energy as sum_i h_i <X_i>."""
    f = (0.5, 0.9, 0.7, 1.1, 0.6, 1.3)
    st = _state(3, 2, D=3, fields=f)
    m = md.TFIM(1.0, 0.9, f)
    a = sp.measure_energy(st, m, bm.BoundaryMPS(200))
    b = dg.measure_energy(st, m, dg.BoundaryMPSDiagonal(200, (100, 100)))
    assert abs(a["energy_total"] - b["energy_total"]) < EXACT * abs(a["energy_total"])
    nw, _ = dg.boundaries(st, dg.BoundaryMPSDiagonal(4, (2, 2)))
    for env in nw:
        for A in env.tensors:
            for leg in (0, 2):
                n0, n1 = A.sector_dims(leg)
                assert n0 <= 2 and n1 <= 2
