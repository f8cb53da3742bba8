"""The stored purified PEPO of the benchmark (8x8 TFIM, h=3.0, beta0 = 0.4,
D=6, chi=36 = 18+18; ``stopeps.jl_b200/states/``) on the GPU.

Its boundary blocks are full rank but their spectra fall by about 1e-5 over
the 18 kept values of a sector, so the subspace iteration of the truncated
SVDs meets columns at the rounding level (on M M^T after two iterations).
The extraction then redoes the plain Cholesky QR with the shift and deflates;
these tests check that no truncated SVD of the contraction falls back to the
full-spectrum Jacobi SVD and that the results still agree with the oracle's
FP64 values (``bench_8x8_D6_chi36_energy.npz``, made by
``tests/golden/make_golden.py``): energy, log norm, <X> sum and per-site <X>
at 1e-10 relative with the exact compression; the zip-up absorption within
the benchmark's 1e-4 energy bar.  Boundary entropies are not recorded here
(``record_boundary_entropy`` needs the full spectrum of every truncation).
"""
import numpy as np
import pytest

from util import golden, rel

pytestmark = pytest.mark.gpu
FIX = "bench_8x8_D6_chi36_energy.npz"
TOL = 1e-10


def _state(sps):
    sites, dims, beta, log_amplitude = sps.bench_states.load()
    e = sps.Engine(8, 8, sps.TFIM(1.0, 3.0), record_boundary_entropy=False)
    st = e.upload_state(sites, dims, True, beta=beta, log_amplitude=log_amplitude)
    return e, st


def _profiled(e, fn):
    e.set_profile(True)
    try:
        out = fn()
        stats = e.kernel_stats()
    finally:
        e.set_profile(False)
    return out, stats


def _jacobi_calls(stats):
    return {k: v for k, v in stats.items() if k.startswith("svd_jacobi")}


def test_purified_energy_exact_compression(sps):
    g = golden(FIX)
    e, st = _state(sps)
    m = sps.BoundaryMPS(36, sps.Z2Space(18, 18))
    en, stats = _profiled(e, lambda: sps.measure_energy(st, m, site_profile=True))
    assert not _jacobi_calls(stats), _jacobi_calls(stats)
    assert any(k.startswith("svd_topk") for k in stats)
    ref = g["energy"]
    assert rel(en["energy_total"], ref[0]) < TOL
    assert rel(en["energy_per_site"], ref[1]) < TOL
    assert rel(en["log_norm"], ref[2]) < TOL
    assert rel(en["x_sum"], ref[3]) < TOL
    np.testing.assert_allclose(en["site_x"], g["site_x"], rtol=TOL, atol=TOL)


def test_purified_zipup_energy_and_draw(sps):
    g = golden(FIX)
    e, st = _state(sps)
    zm = sps.BoundaryMPSZipUp(36, sps.Z2Space(18, 18))
    en, stats = _profiled(e, lambda: sps.measure_energy(st, zm))
    assert not _jacobi_calls(stats), _jacobi_calls(stats)
    de = abs(en["energy_per_site"] - g["energy"][1])
    print(f"zip-up |dE| per site on the purified state: {de:.3e}")
    assert de < 1e-4
    cache = sps.SamplingCache(st, zm)
    u = sps.sample_uniforms(1, 1, 64)
    d, stats = _profiled(e, lambda: sps.sample_configuration(cache, uniforms=u))
    assert not _jacobi_calls(stats), _jacobi_calls(stats)
    # the probability of the drawn configuration, recomputed from it
    d2 = sps.sample_configuration(cache, configuration=d["configuration"])
    assert rel(d2["log_probability"], d["log_probability"]) < 1e-12
