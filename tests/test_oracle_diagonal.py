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


def test_bond_environment_equals_row_environment():
    """``diagonal_update.jl``'s bond environments at exact chi: on every bond of
    a 3x3 D=3 PEPO the reduced metric and the bond hole equal the row
    method's up to the environments' overall scale."""
    from oracle import full_update as fu
    st = _state(3, 3, D=3)
    m = md.TFIM(1.0, 0.9)
    nw, se = dg.boundaries(st, dg.BoundaryMPSDiagonal(400))
    layers = bm.row_layers(st)
    north, south, _ = bm.boundary_environments(layers, bm.BoundaryMPS(400))
    seen = 0
    for t in range(dg.layer_count(3, 3) - 1):
        strip = dg.Strip(st, t, t + 1, nw[t], se[t + 2])
        le, ri = dg.messages(st, strip)
        for direction in ("horizontal", "vertical"):
            for i, j in dg.layer_bonds(3, 3, t, direction):
                a, b = sorted([strip.sites.index(i), strip.sites.index(j)])
                denv = dg.bond_environment(st, strip, le[a], ri[b + 1], i, j, direction)
                renv = bm.bond_environment(st, layers, north, south, i, j, direction)
                pair = fu.reduced_pair(st[i], st[j], md.trotter_gate(m, 3, 3, i, j, 0.05), direction)
                for x, y in ((fu.reduced_metric(renv, pair["Qa"], pair["Qb"]),
                              fu.reduced_metric(denv, pair["Qa"], pair["Qb"])),
                             (bm.bond_hole(renv), dg.bond_hole(denv))):
                    np.testing.assert_allclose(y.a / np.abs(y.a).max(), x.a / np.abs(x.a).max(), atol=1e-13)
                seen += 1
    assert seen == 12


@pytest.mark.parametrize("Lx,Ly", [(3, 3), (2, 3)])
def test_full_update_step_without_truncation_equals_row(Lx, Ly):
    """One second-order step from beta = 0 at D = 4 truncates nothing, so the
    diagonal and row environments give the same state: the same lnZ and energy."""
    from oracle import full_update as fu
    m = md.TFIM(1.0, 0.9)
    out = []
    for method in (bm.BoundaryMPS(400), dg.BoundaryMPSDiagonal(400)):
        st = md.identity_pepo(Lx, Ly)
        md.normalize_state(st)
        r = fu.evolution_step(st, m, 0.05, 4, fu.FullUpdate(), method, record_entropy=True)
        assert r["bond_updates"] == 2 * ((Lx - 1) * Ly + Lx * (Ly - 1))
        e = sp.measure_energy(st, m, bm.BoundaryMPS(400))
        out.append((e["log_norm"], e["energy_per_site"]))
    assert abs(out[0][0] - out[1][0]) < 1e-12 and abs(out[0][1] - out[1][1]) < 1e-12


@pytest.mark.parametrize("h", [0.7, 3.0])
def test_purification_with_diagonal_environments_matches_exact_diagonalization(h):
    """``RunConfig(contraction=BoundaryMPSDiagonal)``: the purification (full
    update and measurement on diagonal boundaries) is within the Trotter error
    of exact diagonalisation and equals the row method's run to 1e-10."""
    out = []
    for diagonal in (False, True):
        c = dr.RunConfig(Lx=3, Ly=2, J=1.0, h=h, beta0=0.2, beta_log=[0.1, 0.2], beta_measure=[0.0, 0.2],
                         delta_tau_pur=0.025, D_pur=4, D_peps=4, chi_environment=16, Ns=4, seed=1,
                         diagonal=diagonal)
        out.append(dr.run_purification(c)[1][-1])
    ex = md.exact_thermal_observables(3, 2, md.TFIM(1.0, h), out[1]["beta"])
    tol = 2e-5 * max(1.0, h * h)
    assert abs(out[1]["lnZ"] - ex["lnZ"]) < tol
    assert abs(out[1]["energy_per_site"] - ex["energy_per_site"]) < tol
    assert abs(out[0]["lnZ"] - out[1]["lnZ"]) < 1e-10
    assert abs(out[0]["energy_per_site"] - out[1]["energy_per_site"]) < 1e-10


def test_forced_repair_on_diagonal_environments_equals_row():
    """update_bond!'s PSD-repair branch forced on every bond: the repaired
    metric comes from the diagonal bond hole, which equals the row hole up to
    scale, so a step without truncation matches the row method's step."""
    from oracle import full_update as fu
    m = md.TFIM(1.0, 0.9)
    bonds = {((x, y), (x + 1, y)) for x in range(2) for y in range(3)}
    bonds |= {((x, y), (x, y + 1)) for x in range(3) for y in range(2)}
    out = []
    for method in (bm.BoundaryMPS(400), dg.BoundaryMPSDiagonal(400)):
        st = md.identity_pepo(3, 3)
        md.normalize_state(st)
        r = fu.evolution_step(st, m, 0.05, 4, fu.FullUpdate(), method, force_repair_bonds=bonds)
        assert r["repairs"] == r["bond_updates"] == 24
        e = sp.measure_energy(st, m, bm.BoundaryMPS(400))
        out.append((e["log_norm"], e["energy_per_site"]))
    assert abs(out[0][0] - out[1][0]) < 1e-11 and abs(out[0][1] - out[1][1]) < 1e-11


@pytest.mark.parametrize("Lx,Ly", [(1, 3), (3, 1), (2, 2)])
def test_physical_kind_on_narrow_lattices(Lx, Ly):
    """The physical kind where layers hold a single site or the frontier
    shrinks to one edge: the same distribution as the row method's at exact chi."""
    st = _state(Lx, Ly)
    cfg0 = [[1 + ((x + y) % 2) for y in range(Ly)] for x in range(Lx)]
    peps, _ = sp.project_configuration(st, cfg0)
    ca = sp.SamplingCache(peps, bm.BoundaryMPS(200), kind="physical")
    cb = dg.DiagonalSamplingCache(peps, dg.BoundaryMPSDiagonal(200), kind="physical")
    total = 0.0
    for cfg in _configs(Lx, Ly):
        p = sp.sample_configuration(ca, configuration=cfg)["log_probability"]
        q = dg.sample_configuration(cb, configuration=cfg)["log_probability"]
        if p == -math.inf:
            assert q == -math.inf
            continue
        assert abs(p - q) < 1e-12
        total += math.exp(q)
    assert abs(total - 1.0) < 1e-12
