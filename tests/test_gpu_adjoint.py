"""The reverse-mode derivative of the row lognorm on the device
(``sps_lognorm_gradient``, ``csrc/adjoint.cu``) against the oracle's
(``oracle/adjoint.py``, pinned on the CPU by finite differences, homogeneity
and the direct <X_i> ratios).

Both canonicalize by full SVDs (the oracle's default gauge) and split the SVD
couplings into broadened 1/(s_j - s_i) and 1/(s_j + s_i) terms; what differs
is the SVD itself (LAPACK against the device's Jacobi), which near-degenerate
singular values turn into differences far below the bar, 1e-7 of each site
gradient's largest entry (the oracle matches central differences to 1e-7 or
better).  Homogeneity (<d lnZ/dA_i, A_i> = 2) holds on the device to 1e-9.
"""
import numpy as np
import pytest

from util import golden, upload_golden, oracle_state

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case,exact", [("pepo_2x3_D2.npz", False), ("pepo_2x3_D2.npz", True),
                                        ("pepo_3x3_D4.npz", False), ("pepo_3x3_D4.npz", True)])
def test_lognorm_gradient_matches_oracle(sps, case, exact):
    from oracle import adjoint as ad
    g = golden(case)
    Lx, Ly = int(g["Lx"]), int(g["Ly"])
    e = sps.Engine(Lx, Ly, sps.TFIM(float(g["J"]), float(g["h"])))
    st = upload_golden(sps, g, e)
    chi, a, b = (int(v) for v in g["chi0"])
    if exact:
        chi, a, b = 256, -1, -1
    m = sps.BoundaryMPS(chi, None if a < 0 else sps.Z2Space(a, b))
    value, grads = sps.lognorm_gradient(st, m)
    ov, og = ad.lognorm_with_gradient(oracle_state(g), chi, None if a < 0 else (a, b))
    assert abs(value - ov) <= 1e-10 * abs(ov)
    sites, _ = st.download()
    for i in range(Lx * Ly):
        x, y = i % Lx, i // Lx
        ref = og[x][y]
        assert np.abs(grads[i] - ref).max() <= 1e-7 * np.abs(ref).max()
        assert abs(float(np.sum(grads[i] * sites[i])) - 2.0) < 1e-9


def test_lognorm_gradient_takes_the_row_method_only(sps):
    g = golden("pepo_2x3_D2.npz")
    e = sps.Engine(int(g["Lx"]), int(g["Ly"]), sps.TFIM(float(g["J"]), float(g["h"])))
    st = upload_golden(sps, g, e)
    for m in (sps.BoundaryMPSDiagonal(4), sps.BoundaryMPSRowVariational(4)):
        with pytest.raises(sps._lib.EngineError):
            sps.lognorm_gradient(st, m)
    value, _ = sps.lognorm_gradient(st, sps.BoundaryMPS(4))
    assert np.isfinite(value)


def test_row_checkpoints_give_the_same_derivative(sps):
    """With per-row checkpoints the reverse pass recomputes each row's
    factorizations from its incoming boundary: the same operations on the same
    boundary, so the derivative agrees with the full tape to roundoff (bar
    1e-8 of the largest entry: the large-block SVD sums with floating-point
    atomics, whose order may differ between the two passes)."""
    g = golden("pepo_3x3_D4.npz")
    e = sps.Engine(3, 3, sps.TFIM(float(g["J"]), float(g["h"])))
    st = upload_golden(sps, g, e)
    chi, a, b = (int(v) for v in g["chi0"])
    m = sps.BoundaryMPS(chi, sps.Z2Space(a, b))
    v0, g0 = sps.lognorm_gradient(st, m)
    v1, g1 = sps.lognorm_gradient(st, m, checkpoint_rows=True)
    assert abs(v1 - v0) <= 1e-12 * abs(v0)
    for x0, x1 in zip(g0, g1):
        assert np.abs(x1 - x0).max() <= 1e-8 * np.abs(x0).max()


def test_field_gradient_matches_direct_ratios_and_oracle(sps):
    """<X_i> from one reverse pass against the direct per-site ratios of
    measure_energy at exact chi (1e-9; at truncating chi the two routes
    differ by the truncation), and d lnZ/dh_i = beta <X_i> against the
    oracle's reverse pass at chi0 on the 3x3 D=4 fixture (1e-7 relative, the
    bar of the site gradients it contracts)."""
    from oracle import adjoint as ad
    g = golden("pepo_2x3_D2.npz")
    e = sps.Engine(int(g["Lx"]), int(g["Ly"]), sps.TFIM(float(g["J"]), float(g["h"])))
    st = upload_golden(sps, g, e)
    m = sps.BoundaryMPS(256)
    r = sps.lognorm_field_gradient(st, m)
    direct = sps.measure_energy(st, m)["site_x"]
    assert np.abs(r["site_x"] - direct).max() < 1e-9
    assert np.allclose(r["d_fields"], float(g["beta"]) * r["site_x"].T.reshape(-1), rtol=0, atol=1e-15)

    g = golden("pepo_3x3_D4.npz")
    e = sps.Engine(3, 3, sps.TFIM(float(g["J"]), float(g["h"])))
    st = upload_golden(sps, g, e)
    chi, a, b = (int(v) for v in g["chi0"])
    r = sps.lognorm_field_gradient(st, sps.BoundaryMPS(chi, sps.Z2Space(a, b)), checkpoint_rows=True)
    ov, osx, odf = ad.field_gradient(oracle_state(g), chi, (a, b))
    assert abs(r["log_norm"] - ov) <= 1e-10 * abs(ov)
    assert np.abs(r["d_fields"] - odf).max() <= 1e-7 * np.abs(odf).max()


def test_autograd_function_on_the_device(sps):
    """torch.autograd through LognormFunction returns the device derivative
    scaled by the cotangent."""
    import torch
    g = golden("pepo_2x3_D2.npz")
    e = sps.Engine(int(g["Lx"]), int(g["Ly"]), sps.TFIM(float(g["J"]), float(g["h"])))
    st = upload_golden(sps, g, e)
    sites, dims = st.download()
    m = sps.BoundaryMPS(4)
    value, ref = sps.lognorm_gradient(st, m)
    ts = [torch.tensor(s, dtype=torch.float64, requires_grad=True) for s in sites]
    out = sps.lognorm_differentiable(e, ts, dims, m, beta=float(g["beta"]), log_amplitude=float(g["log_amplitude"]))
    assert abs(out.item() - value) <= 1e-13 * abs(value)
    grads = torch.autograd.grad(-2.0 * out, ts)
    for a, b in zip(grads, ref):
        assert np.abs(a.numpy() + 2.0 * b).max() <= 1e-12 * np.abs(b).max()


def test_lognorm_gradient_at_the_differentiation_shape(sps):
    """6x6 D=4 chi=24 (12+12), a seeded synthetic PEPO at beta 1 whose
    boundary blocks are numerically rank deficient: the device derivative
    against the oracle's (which matches central differences to 1.5e-7 there),
    1e-6 of each site gradient's largest entry, homogeneity to 1e-9."""
    from oracle import adjoint as ad
    from oracle.model import State
    from oracle.z2 import T, leg
    L = 6
    sites, dims = sps.synthetic.synthetic_pepo(L, L, 4, 0.3, 7)
    e = sps.Engine(L, L, sps.TFIM(1.0, 3.0))
    st = e.upload_state(sites, dims, True, beta=1.0)
    value, grads = sps.lognorm_gradient(st, sps.BoundaryMPS(24, sps.Z2Space(12, 12)), checkpoint_rows=True)
    d = np.asarray(dims).reshape(L * L, 6, 2)
    S = [[None] * L for _ in range(L)]
    for i in range(L * L):
        S[i % L][i // L] = T(np.asarray(sites[i]).reshape([int(a + b) for a, b in d[i]]),
                             [leg(int(a), int(b)) for a, b in d[i]])
    ov, og = ad.lognorm_with_gradient(State(L, L, S, 1.0, 0.0, "pepo"), 24, (12, 12))
    assert abs(value - ov) <= 1e-10 * abs(ov)
    for i in range(L * L):
        ref = og[i % L][i // L]
        assert np.abs(grads[i] - ref).max() <= 1e-6 * np.abs(ref).max()
        assert abs(float(np.sum(grads[i] * np.asarray(sites[i]).reshape(ref.shape))) - 2.0) < 1e-9
