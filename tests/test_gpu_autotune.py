"""The autotuner: launch shapes picked by timing on first use, shared by every
engine of the process, results unchanged beyond rounding."""
import numpy as np
import pytest

from util import golden, upload_golden, rel

pytestmark = pytest.mark.gpu


def test_autotuned_contractions_match_and_are_recorded(sps):
    g = golden("pepo_4x4_D4.npz")
    e = sps.Engine(int(g["Lx"]), int(g["Ly"]), sps.TFIM(float(g["J"]), float(g["h"])))
    st = upload_golden(sps, g, e)
    m = sps.BoundaryMPS(int(g["chi0"][0]), sps.Z2Space(int(g["chi0"][1]), int(g["chi0"][2])))
    ref = sps.measure_energy(st, m)
    e.set_autotune(True)
    try:
        tuned = sps.measure_energy(st, m)
        again = sps.measure_energy(st, m)   # every shape tuned by now: no timing runs
        report = e.autotune_report()
    finally:
        e.set_autotune(False)
    assert any(k.split(":")[1] == "gemm_gather.split" for k in report), report
    for k, v in report.items():
        assert v["choice"] in [int(c) for c in v["ms"]]
    assert rel(tuned["energy_per_site"], ref["energy_per_site"]) < 1e-12
    assert tuned["energy_per_site"] == again["energy_per_site"]
    assert rel(tuned["energy_per_site"], float(g["energy0"][1])) < 1e-10


def test_autotuned_tensor_core_tile(sps):
    e = sps.Engine(2, 2)
    e.set_autotune(True)
    rng = np.random.default_rng(5)
    a = rng.standard_normal((700, 900))
    b = rng.standard_normal((900, 500))
    c, _ = e.la_gemm_mixed(a, b, "3xtf32")
    e.set_autotune(False)
    report = e.autotune_report()
    keys = [k for k in report if ":tc_gemm.bn:" in k]
    assert keys, report
    assert report[keys[0]]["choice"] in (64, 128, 256)
    assert np.linalg.norm(c - a @ b) / np.linalg.norm(a @ b) < 1e-4   # split TF32, FP32 accumulation
