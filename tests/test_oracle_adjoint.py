"""The oracle's reverse-mode derivative of the row boundary-MPS lognorm
(``oracle/adjoint.py``: QR / LQ and truncated-SVD backward per parity block,
Lorentzian-broadened) pinned on the CPU.

* central finite differences (step 1e-5) of lognorm along a random
  direction in every site tensor, at exact and truncating chi;
* homogeneity: lognorm grows by 2 log c when one site tensor is scaled by c,
  so <dlnZ/dA_i, A_i> = 2 for every site, truncation included;
* the direct ratios: the derivative along an X insertion on the ket's
  physical leg is 2 <X_i>, the per-site value ``measure_energy`` reports.
"""
import copy

import numpy as np
import pytest

from oracle import adjoint as ad, boundary as bm, driver as dr, model as md, sampling as sp, z2
from oracle.z2 import T


def _state(Lx, Ly, D=3, beta=0.3, h=1.0):
    c = dr.RunConfig(Lx=Lx, Ly=Ly, J=1.0, h=h, beta0=beta, beta_log=[beta], beta_measure=[beta],
                     delta_tau_pur=0.05, D_pur=D, D_peps=D, chi_environment=64, Ns=1)
    return dr.run_purification(c)[0]


def _shifted(st, dirs, eps):
    s2 = copy.copy(st)
    s2.sites = [[T(st[x, y].a + eps * dirs[x][y], st[x, y].p) for y in range(st.Ly)] for x in range(st.Lx)]
    return s2


@pytest.mark.parametrize("Lx,Ly,D,chi", [(3, 2, 2, 64), (3, 3, 3, 64), (3, 3, 3, 6), (4, 3, 3, 5)])
def test_gradient_matches_finite_differences(Lx, Ly, D, chi):
    st = _state(Lx, Ly, D)
    value, g = ad.lognorm_with_gradient(st, chi)
    ref = bm.lognorm(st, bm.BoundaryMPS(chi))["log_norm"]
    assert abs(value - ref) <= 1e-13 * abs(ref)
    rng = np.random.default_rng(Lx * 10 + chi)
    dirs = [[rng.standard_normal(st[x, y].shape) * z2.parity_mask(st[x, y].p) for y in range(Ly)]
            for x in range(Lx)]
    eps = 1e-5
    up = bm.lognorm(_shifted(st, dirs, eps), bm.BoundaryMPS(chi))["log_norm"]
    down = bm.lognorm(_shifted(st, dirs, -eps), bm.BoundaryMPS(chi))["log_norm"]
    fd = (up - down) / (2 * eps)
    adj = sum(float(np.sum(g[x][y] * dirs[x][y])) for x in range(Lx) for y in range(Ly))
    assert abs(fd - adj) <= 1e-7 * abs(fd)
    for x in range(Lx):
        for y in range(Ly):
            assert abs(float(np.sum(g[x][y] * st[x, y].a)) - 2.0) < 1e-12


def test_gradient_along_x_insertions_is_twice_the_site_magnetisation():
    st = _state(3, 3)
    X, _, _ = md.spin_operators()
    _, g = ad.lognorm_with_gradient(st, 400)
    e = sp.measure_energy(st, md.TFIM(1.0, 1.0), bm.BoundaryMPS(400))
    for x in range(3):
        for y in range(3):
            XA = np.einsum("pu,wnuaes->wnpaes", X, st[x, y].a)
            assert abs(float(np.sum(g[x][y] * XA)) / 2 - e["site_x"][x, y]) < 1e-10


def test_field_gradient_matches_finite_differences_of_the_purification():
    """d lnZ/dh_i = beta <X_i> from one reverse pass against the central
    difference (step 1e-4) of the purified lnZ in each site's field, on a 2x2
    (exact chi): the Trotterized state is exp(-beta H_eff / 2) with H_eff
    = H + O(delta_tau^2), so the two differ by the Trotter error alone,
    measured 5.2e-6, 1.2e-6 and 2.2e-7 at delta_tau 0.025, 0.0125 and
    0.00625 (the last is tested).  <X_i> from the reverse pass equals the
    direct per-site ratio to 1e-10."""
    rng = np.random.default_rng(7)
    fields = tuple(3.0 + rng.uniform(-0.05, 0.05, 4))

    def run(f):
        c = dr.RunConfig(Lx=2, Ly=2, J=1.0, h=3.0, fields=f, beta0=0.2, beta_log=[0.2], beta_measure=[0.2],
                         delta_tau_pur=0.00625, D_pur=4, D_peps=4, chi_environment=16, Ns=1)
        return dr.run_purification(c)

    st, rows = run(fields)
    value, site_x, d_fields = ad.field_gradient(st, 16)
    assert abs(value - rows[-1]["lnZ"]) < 1e-12 * abs(value)
    e = sp.measure_energy(st, md.TFIM(1.0, 3.0, fields), bm.BoundaryMPS(16))
    assert np.abs(site_x - e["site_x"]).max() < 1e-10
    step = 1e-4
    for i in range(4):
        lz = []
        for s in (+1, -1):
            f = list(fields)
            f[i] += s * step
            lz.append(run(tuple(f))[1][-1]["lnZ"])
        assert abs((lz[0] - lz[1]) / (2 * step) - d_fields[i]) < 5e-7


@pytest.mark.parametrize("case", ["pepo_2x3_D2.npz", "pepo_3x3_D4.npz"])
def test_svd_gauge_of_the_canonical_sweep_gives_the_same_derivative(case):
    """The device canonicalizes by full SVDs (L = U S, Q = V^T) where the
    reference takes LQs.  The truncated boundary does not depend on that
    gauge, and the derivative agrees up to the Lorentzian broadening's
    gauge dependence: 2e-16 on the 2x3 D=2 fixture, 2.3e-9 of each site
    gradient's largest entry on the 3x3 D=4 one (bar 1e-8), exact chi and
    chi0 alike."""
    from util import golden, oracle_state
    g = golden(case)
    st = oracle_state(g)
    chi, a, b = (int(v) for v in g["chi0"])
    for c, sp_ in ((chi, None if a < 0 else (a, b)), (256, None)):
        v1, g1 = ad.lognorm_with_gradient(st, c, sp_)
        v2, g2 = ad.lognorm_with_gradient(st, c, sp_, canonical="svd")
        assert abs(v1 - v2) < 1e-13 * abs(v1)
        for x in range(st.Lx):
            for y in range(st.Ly):
                assert np.abs(g1[x][y] - g2[x][y]).max() <= 1e-8 * np.abs(g1[x][y]).max()
                assert abs(float(np.sum(g2[x][y] * st[x, y].a)) - 2.0) < 1e-12


@pytest.mark.parametrize("Lx,Ly,D,chi,space", [(3, 3, 3, 6, (3, 3)), (4, 3, 3, 8, (5, 3))])
def test_gradient_with_a_sector_budget_matches_finite_differences(Lx, Ly, D, chi, space):
    """truncrank & truncspace: the kept set of each truncated SVD is a prefix
    of each parity block under the sector budget; central differences agree
    to 7e-10 and 5e-9 relative here (bar 1e-7)."""
    st = _state(Lx, Ly, D)
    value, g = ad.lognorm_with_gradient(st, chi, space)
    ref = bm.lognorm(st, bm.BoundaryMPS(chi, space))["log_norm"]
    assert abs(value - ref) <= 1e-13 * abs(ref)
    rng = np.random.default_rng(3)
    dirs = [[rng.standard_normal(st[x, y].shape) * z2.parity_mask(st[x, y].p) for y in range(Ly)]
            for x in range(Lx)]
    eps = 1e-5
    up = bm.lognorm(_shifted(st, dirs, eps), bm.BoundaryMPS(chi, space))["log_norm"]
    down = bm.lognorm(_shifted(st, dirs, -eps), bm.BoundaryMPS(chi, space))["log_norm"]
    fd = (up - down) / (2 * eps)
    adj = sum(float(np.sum(g[x][y] * dirs[x][y])) for x in range(Lx) for y in range(Ly))
    assert abs(fd - adj) <= 1e-7 * abs(fd)


@pytest.mark.parametrize("chi,space", [(256, None), (24, (12, 12))])
def test_gradient_on_rank_deficient_boundaries(sps, chi, space):
    """A seeded synthetic 4x4 D=4 PEPO, whose absorbed boundaries have
    numerically rank-deficient blocks: the SVD gauge with the split,
    broadened couplings matches central differences to 7e-10 and 6e-10
    (bar 1e-8); the LQ gauge, whose reverse rule solves with L, is off by
    1e-4 there (not tested)."""
    from oracle.model import State
    from oracle.z2 import leg
    sites, dims = sps.synthetic.synthetic_pepo(4, 4, 4, 0.3, 7)
    dims = np.asarray(dims).reshape(16, 6, 2)
    S = [[None] * 4 for _ in range(4)]
    for i in range(16):
        S[i % 4][i // 4] = T(np.asarray(sites[i]).reshape([int(a + b) for a, b in dims[i]]),
                             [leg(int(a), int(b)) for a, b in dims[i]])
    st = State(4, 4, S, 1.0, 0.0, "pepo")
    value, g = ad.lognorm_with_gradient(st, chi, space)
    rng = np.random.default_rng(11)
    dirs = [[rng.standard_normal(st[x, y].shape) * (st[x, y].a != 0) for y in range(4)] for x in range(4)]
    eps = 1e-6
    up = bm.lognorm(_shifted(st, dirs, eps), bm.BoundaryMPS(chi, space))["log_norm"]
    down = bm.lognorm(_shifted(st, dirs, -eps), bm.BoundaryMPS(chi, space))["log_norm"]
    fd = (up - down) / (2 * eps)
    adj = sum(float(np.sum(g[x][y] * dirs[x][y])) for x in range(4) for y in range(4))
    assert abs(fd - adj) <= 1e-8 * abs(fd)
    for x in range(4):
        for y in range(4):
            assert abs(float(np.sum(g[x][y] * st[x, y].a)) - 2.0) < 1e-12


def test_gradient_at_the_differentiation_shape(sps):
    """The 6x6 D=4 chi=24 (12+12) shape of the differentiation workload, on a
    seeded synthetic PEPO at beta 1: the derivative along a random direction
    matches central differences (step 1e-5) to 1.5e-7 relative (bar 1e-6)."""
    from oracle.model import State
    from oracle.z2 import leg
    L = 6
    sites, dims = sps.synthetic.synthetic_pepo(L, L, 4, 0.3, 7)
    dims = np.asarray(dims).reshape(L * L, 6, 2)
    S = [[None] * L for _ in range(L)]
    for i in range(L * L):
        S[i % L][i // L] = T(np.asarray(sites[i]).reshape([int(a + b) for a, b in dims[i]]),
                             [leg(int(a), int(b)) for a, b in dims[i]])
    st = State(L, L, S, 1.0, 0.0, "pepo")
    value, g = ad.lognorm_with_gradient(st, 24, (12, 12))
    rng = np.random.default_rng(11)
    dirs = [[rng.standard_normal(st[x, y].shape) * (st[x, y].a != 0) for y in range(L)] for x in range(L)]
    eps = 1e-5
    up = bm.lognorm(_shifted(st, dirs, eps), bm.BoundaryMPS(24, (12, 12)))["log_norm"]
    down = bm.lognorm(_shifted(st, dirs, -eps), bm.BoundaryMPS(24, (12, 12)))["log_norm"]
    fd = (up - down) / (2 * eps)
    adj = sum(float(np.sum(g[x][y] * dirs[x][y])) for x in range(L) for y in range(L))
    assert abs(fd - adj) <= 1e-6 * abs(fd)
