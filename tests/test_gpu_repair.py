"""update_bond!'s PSD-repair branch (``full_update.jl:490-501``, the repaired
metric of ``_positive_reduced_metric`` :278-340) forced on every bond of one
step of the 3x3 D=4 PEPS, against the oracle with the same bonds forced: the
bond holes' parity blocks reach 512 rows here (32 in the 2x3 D=2 case of
``test_gpu_batch.py``), through the single-CTA eigendecomposition and, with a
lowered threshold, the multi-CTA route of large holes.
"""
import numpy as np
import pytest

from util import golden, upload_golden, oracle_state, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("multi_cta", [False, True])
def test_forced_psd_repair_at_d4_matches_oracle(sps, multi_cta):
    from oracle import full_update as fu, model as md, boundary as bm, sampling as osp
    g = golden("pepo_3x3_D4.npz")
    e = sps.Engine(3, 3, sps.TFIM(float(g["J"]), float(g["h"])))
    st = upload_golden(sps, g, e)
    pc = g["peps_cfg"]
    D = int(pc[0])
    space = None if pc[1] < 0 else (int(pc[1]), int(pc[2]))
    chi, a, b = int(pc[3]), int(pc[4]), int(pc[5])
    m = sps.BoundaryMPS(chi, None if a < 0 else sps.Z2Space(a, b))
    cfg = g["configs"][0]
    ps, _ = sps.project_configuration(st, cfg)
    e.set_injection(force_repair=True, multi_cta_eigh_min=64 if multi_cta else 0)
    try:
        r = sps.evolution_step(ps, float(g["dtau"]), D, m, None if space is None else sps.Z2Space(*space))
    finally:
        e.set_injection()
    assert r["repairs"] == r["bond_updates"] == 24
    ops, _ = osp.project_configuration(oracle_state(g), np.asarray(cfg).tolist())
    bonds = {((x, y), (x + 1, y)) for x in range(2) for y in range(3)}
    bonds |= {((x, y), (x, y + 1)) for x in range(3) for y in range(2)}
    om = bm.BoundaryMPS(chi, None if a < 0 else (a, b))
    model = md.TFIM(float(g["J"]), float(g["h"]))
    ro = fu.evolution_step(ops, model, float(g["dtau"]), D, fu.FullUpdate(), om, space=space,
                           force_repair_bonds=bonds)
    assert ro["repairs"] == r["repairs"]
    assert rel(r["log_normalization_sum"], sum(v for _, v in ro["normalizations"])) < 1e-9
    en = sps.measure_energy(ps, m)
    oen = osp.measure_energy(ops, model, om)
    assert rel(en["energy_per_site"], oen["energy_per_site"]) < 1e-9
