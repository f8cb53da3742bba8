"""The mixed-precision contraction path (tcgen05 GEMM) against FP64.

``sps_set_precision`` routes the large contraction GEMMs to the tcgen05
tensor cores (TF32, 3xTF32 or 3xBF16 operands, FP32 accumulation) while the
truncations, normalisations and log-weights stay FP64.  The GEMM itself is
checked against NumPy FP64 with per-mode error bounds; the physics at the
headline shapes (4x4 lattice, D=6, chi=36) against the FP64 oracle fixture:
energy per site and magnetisation of the beta0 state and after one
full-update step, and the Born draws.  The bounds are the accuracy of each
arithmetic (relative Frobenius error of a GEMM; absolute error of per-site
observables), far above FP64 rounding and far below the 1e-4 energy target.
"""
import numpy as np
import pytest

from util import golden, rel

pytestmark = pytest.mark.gpu

# relative Frobenius error of one GEMM, per mode: the operand rounding (TF32
# 2^-11; split TF32 ~2^-21; split BF16 ~2^-16 per product) plus the FP32
# accumulation over K, which dominates the split TF32 mode (~2^-24 sqrt(K) to
# 2^-24 K: 4e-6 at K = 700, 3e-5 at K = 4096 measured on the B200)
GEMM_TOL = {"tf32": 3e-3, "3xtf32": 1e-4, "3xbf16": 2e-4}
# absolute error of the energy / magnetisation per site at the headline shapes:
# the split modes within the 1e-4 energy target with a factor-two margin, the
# single-pass TF32 mode (2^-11 per operand) an order of magnitude looser
OBS_TOL = {"tf32": 2e-3, "3xtf32": 5e-5, "3xbf16": 5e-5}
CASE = "headline_4x4_D6_chi36.npz"


@pytest.mark.parametrize("mode", ["tf32", "3xtf32", "3xbf16"])
@pytest.mark.parametrize("m,n,k", [(300, 200, 700), (128, 128, 64), (1000, 37, 513), (65, 300, 4096)])
def test_tc_gemm_against_numpy(sps, mode, m, n, k):
    e = sps.Engine(2, 2)
    rng = np.random.default_rng(m + 7 * n + 13 * k)
    a = rng.standard_normal((m, k))
    b = rng.standard_normal((k, n))
    c, ms = e.la_gemm_mixed(a, b, mode)
    ref = a @ b
    err = np.linalg.norm(c - ref) / np.linalg.norm(ref)
    assert err < GEMM_TOL[mode], (mode, err)
    # a second call reuses the pooled workspace and gives the same result
    c2, _ = e.la_gemm_mixed(a, b, mode)
    np.testing.assert_array_equal(c, c2)


def _headline(sps):
    g = golden(CASE)
    e = sps.Engine(int(g["Lx"]), int(g["Ly"]), sps.TFIM(float(g["J"]), float(g["h"])))
    L = int(g["Lx"]) * int(g["Ly"])
    dims = g["dims"].reshape(L, 6, 2)
    sites, off = [], 0
    for i in range(L):
        n = int(np.prod([a + b for a, b in dims[i]]))
        sites.append(g["data"][off:off + n])
        off += n
    st = e.upload_state(sites, dims, True, beta=float(g["beta"]), log_amplitude=float(g["log_amplitude"]))
    return g, e, st


@pytest.mark.parametrize("mode", ["tf32", "3xtf32", "3xbf16"])
def test_mixed_precision_observables_against_fp64_oracle(sps, mode):
    g, e, st = _headline(sps)
    chi, a, b = (int(v) for v in g["chi"])
    m = sps.BoundaryMPS(chi, sps.Z2Space(a, b))
    L = int(g["Lx"]) * int(g["Ly"])
    e.set_precision(mode)
    e.set_profile(True)
    try:
        en = sps.measure_energy(st, m, site_profile=True)
        stats = e.kernel_stats()
    finally:
        e.set_profile(False)
        e.set_precision("fp64")
    assert any(k.startswith("tc_gemm") for k in stats), "no contraction took the tensor-core path"
    ref = g["plain_energy"]
    de = abs(en["energy_per_site"] - ref[1])
    dm = abs(en["x_sum"] - ref[3]) / L
    print(f"{mode}: |dE| per site {de:.3e}, |dM| per site {dm:.3e}")
    assert de < OBS_TOL[mode]
    assert dm < OBS_TOL[mode]
    assert rel(en["log_norm"], ref[2]) < 50 * OBS_TOL[mode]


@pytest.mark.parametrize("mode", ["3xtf32", "3xbf16"])
def test_mixed_precision_draws_and_full_update_step(sps, mode):
    """Born draws (zip-up cache) and one full-update step of the projected D=6
    PEPS in the mixed mode, against the FP64 oracle: identical configurations,
    log-probabilities and the post-step energy within the mode's accuracy."""
    g, e, st = _headline(sps)
    chi, a, b = (int(v) for v in g["chi"])
    e.set_precision(mode)
    try:
        cache = sps.SamplingCache(st, sps.BoundaryMPSZipUp(chi, sps.Z2Space(a, b)))
        for u, cfg, lp in zip(g["uniforms"], g["zip_configs"], g["zip_log_probs"]):
            d = sps.sample_configuration(cache, uniforms=u)
            np.testing.assert_array_equal(d["configuration"], cfg)
            assert abs(d["log_probability"] - lp) < 100 * OBS_TOL[mode]
        m = sps.BoundaryMPS(chi, sps.Z2Space(a, b))
        ps, _ = sps.project_configuration(st, g["plain_configs"][0])
        D = int(g["D"])
        r = sps.evolution_step(ps, float(g["dtau"]), D, m, sps.Z2Space(D // 2, D // 2))
        en = sps.measure_energy(ps, m)
    finally:
        e.set_precision("fp64")
    assert r["bond_updates"] == int(g["step_report"][3])
    de = abs(en["energy_per_site"] - g["step_energy"][0])
    print(f"{mode}: after one FU step |dE| per site {de:.3e}")
    assert de < 10 * OBS_TOL[mode]
