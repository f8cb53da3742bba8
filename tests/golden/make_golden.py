"""Generate the golden fixtures of the parity tests from the CPU oracle.

The reference (StoPEPS.jl) cannot run here (no Julia), so every fixture is an
output of the oracle restatement under ``oracle/``; the oracle itself is
pinned against exact diagonalization in ``tests/test_oracle.py``.
Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import driver as dr, model as md, sampling as sp, boundary as bm, full_update as fu  # noqa: E402
from oracle.z2 import T  # noqa: E402


def state_arrays(st):
    """Flatten an oracle state (x + y*Lx order) into data + per-leg (n0, n1)."""
    data, dims = [], []
    for y in range(st.Ly):
        for x in range(st.Lx):
            t = st[x, y]
            for p in t.p:
                n0 = int((p == 0).sum())
                assert np.all(p[:n0] == 0) and np.all(p[n0:] == 1), "site legs must be sector sorted"
                dims.append((n0, len(p) - n0))
            data.append(t.a.reshape(-1))
    return np.concatenate(data), np.asarray(dims, np.int32).reshape(st.Lx * st.Ly, 6, 2)


def pepo_case(name, Lx, Ly, h, D, space, chi_env, env_space, beta0, dtau, chis, peps_D, peps_space, peps_chi,
              peps_env_space, ndraws=4, seed=1, update=None):
    c = dr.RunConfig(Lx=Lx, Ly=Ly, J=1.0, h=h, beta0=beta0, beta_log=[beta0], beta_measure=[beta0],
                     delta_tau_pur=dtau, delta_tau_peps=dtau, D_pur=D, D_peps=D, bond_space_pur=space,
                     bond_space_peps=space, chi_environment=chi_env, environment_space=env_space, Ns=1, seed=seed,
                     record_boundary_entropy=True, update=update or fu.FullUpdate())
    st, rows = dr.run_purification(c)
    data, dims = state_arrays(st)
    out = dict(Lx=Lx, Ly=Ly, J=1.0, h=h, beta=st.beta, log_amplitude=st.log_amplitude, data=data, dims=dims,
               pur_lnZ=rows[-1]["lnZ"], pur_energy=rows[-1]["energy_per_site"])
    model = md.TFIM(1.0, h)
    for k, (chi, csp) in enumerate(chis):
        m = bm.BoundaryMPS(chi, csp)
        ln = bm.lognorm(st, m)
        en = sp.measure_energy(st, model, m, record_entropy=True)
        out[f"chi{k}"] = np.array([chi, -1 if csp is None else csp[0], -1 if csp is None else csp[1]])
        out[f"lognorm{k}"] = np.array([ln["log_norm"], ln["tensor_log_norm"], ln["max_environment_truncation"]])
        out[f"energy{k}"] = np.array([en["energy_total"], en["energy_per_site"], en["log_norm"], en["x_sum"],
                                      en["max_environment_truncation"]])
        out[f"site_x{k}"] = en["site_x"]
    # Born draws at the first chi
    chi, csp = chis[0]
    cache = sp.SamplingCache(st, bm.BoundaryMPS(chi, csp))
    U = np.stack([dr.sample_uniforms(seed, i, Lx * Ly) for i in range(1, ndraws + 1)])
    cfgs, lps = [], []
    for u in U:
        d = sp.sample_configuration(cache, uniforms=u)
        cfgs.append(np.asarray(d["configuration"]))
        lps.append(d["log_probability"])
    out.update(uniforms=U, configs=np.stack(cfgs), log_probs=np.asarray(lps))
    # projection of draw 1, its energy, one PEPS evolution step and its energy
    ps, norms = sp.project_configuration(st, cfgs[0].tolist())
    pm = bm.BoundaryMPS(peps_chi, peps_env_space)
    e0 = sp.measure_energy(ps, model, pm)
    r = fu.evolution_step(ps, model, dtau, peps_D, update or fu.FullUpdate(), pm, space=peps_space,
                          record_entropy=True)
    e1 = sp.measure_energy(ps, model, pm)
    out.update(proj_norms=np.asarray([v for _, v in norms]),
               proj_energy=np.array([e0["energy_per_site"], e0["log_norm"], e0["x_sum"]]),
               step_norm_sum=sum(v for _, v in r["normalizations"]),
               step_report=np.array([r["max_state_truncation"], r["max_environment_truncation"],
                                     r["max_boundary_entropy"], r["bond_updates"]]),
               step_stops=np.array([r["stop_reasons"][k] for k in
                                    ("error_tolerance", "iteration_limit", "residual_fallback", "disabled")]),
               step_energy=np.array([e1["energy_per_site"], e1["log_norm"], e1["tensor_log_norm"], e1["x_sum"]]),
               peps_cfg=np.array([peps_D, -1 if peps_space is None else peps_space[0],
                                  -1 if peps_space is None else peps_space[1], peps_chi,
                                  -1 if peps_env_space is None else peps_env_space[0],
                                  -1 if peps_env_space is None else peps_env_space[1]]),
               dtau=dtau)
    np.savez_compressed(os.path.join(HERE, name), **out)
    print(name, "pur lnZ", out["pur_lnZ"], "E", out["pur_energy"], "draw logp", out["log_probs"],
          "step", out["step_stops"], out["step_report"])


def synthetic_state(Lx, Ly, D, eps, seed):
    """The seeded synthetic PEPO of ``stopeps.jl_b200/synthetic.py`` (pure NumPy)
    as an oracle state; loaded from the file so that no device code is imported."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_synthetic", os.path.join(ROOT, "stopeps.jl_b200", "synthetic.py"))
    syn = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(syn)
    from oracle.model import State
    from oracle.z2 import leg
    sites, dims = syn.synthetic_pepo(Lx, Ly, D, eps, seed)
    grid = [[None] * Ly for _ in range(Lx)]
    for i, (a, d) in enumerate(zip(sites, dims)):
        grid[i % Lx][i // Lx] = T(np.asarray(a, float), [leg(int(p), int(q)) for p, q in d])
    return State(Lx, Ly, grid, 0.4, 0.0, "pepo")


def headline_case(name, Lx=4, Ly=4, D=6, chi=36, h=3.0, dtau=0.02, ndraws=3, seed=1):
    """The headline shapes (D=6 = 3+3, chi=36 = 18+18, h=3.0, tau=0.02) on a
    small lattice: the seeded synthetic beta0 PEPO of the benchmark workload.
    Both absorptions (exact compression and zip-up): lognorm, energy with the
    site <X> profile and the Schmidt entropies, Born draws; the projection of
    the first draw and one full-update step of that D=6 PEPS."""
    st = synthetic_state(Lx, Ly, D, 0.15, 7)
    data, dims = state_arrays(st)
    model = md.TFIM(1.0, h)
    sec = (chi // 2, chi // 2)
    out = dict(Lx=Lx, Ly=Ly, J=1.0, h=h, beta=st.beta, log_amplitude=st.log_amplitude, data=data, dims=dims,
               chi=np.array([chi, sec[0], sec[1]]), dtau=dtau, D=D)
    U = np.stack([dr.sample_uniforms(seed, i, Lx * Ly) for i in range(1, ndraws + 1)])
    out["uniforms"] = U
    for tag, zipup in (("plain", False), ("zip", True)):
        m = bm.BoundaryMPS(chi, sec, zipup=zipup)
        ln = bm.lognorm(st, m)
        en = sp.measure_energy(st, model, m, record_entropy=not zipup)
        out[f"{tag}_lognorm"] = np.array([ln["log_norm"], ln["tensor_log_norm"], ln["max_environment_truncation"]])
        out[f"{tag}_energy"] = np.array([en["energy_total"], en["energy_per_site"], en["log_norm"], en["x_sum"],
                                         en["max_environment_truncation"], en["zz_sum"]])
        out[f"{tag}_site_x"] = en["site_x"]
        if not zipup:
            out["plain_Se_north"] = en["Se"]["north"]
            out["plain_Se_south"] = en["Se"]["south"]
        cache = sp.SamplingCache(st, m)
        cfgs, lps = [], []
        for u in U:
            d = sp.sample_configuration(cache, uniforms=u)
            cfgs.append(np.asarray(d["configuration"]))
            lps.append(d["log_probability"])
        out[f"{tag}_configs"] = np.stack(cfgs)
        out[f"{tag}_log_probs"] = np.asarray(lps)
        print(name, tag, "lognorm", ln["log_norm"], "E", en["energy_per_site"], "logp", lps, flush=True)
    cfg0 = out["plain_configs"][0]
    ps, norms = sp.project_configuration(st, cfg0.tolist())
    pm = bm.BoundaryMPS(chi, sec)
    e0 = sp.measure_energy(ps, model, pm)
    r = fu.evolution_step(ps, model, dtau, D, fu.FullUpdate(), pm, space=(D // 2, D // 2), record_entropy=True)
    e1 = sp.measure_energy(ps, model, pm)
    out.update(proj_norms=np.asarray([v for _, v in norms]),
               proj_energy=np.array([e0["energy_per_site"], e0["log_norm"], e0["x_sum"]]),
               step_norm_sum=sum(v for _, v in r["normalizations"]),
               step_norms=np.asarray([v for _, v in r["normalizations"]]),
               step_report=np.array([r["max_state_truncation"], r["max_environment_truncation"],
                                     r["max_boundary_entropy"], r["bond_updates"]]),
               step_stops=np.array([r["stop_reasons"][k] for k in
                                    ("error_tolerance", "iteration_limit", "residual_fallback", "disabled")]),
               step_energy=np.array([e1["energy_per_site"], e1["log_norm"], e1["tensor_log_norm"], e1["x_sum"]]),
               step_site_x=e1["site_x"])
    np.savez_compressed(os.path.join(HERE, name), **out)
    print(name, "step", out["step_stops"], out["step_report"], "E1", e1["energy_per_site"], flush=True)


def stored_state(name):
    """A stored PEPO of ``stopeps.jl_b200/bench_states.py`` as an oracle state."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_bench_states",
                                                  os.path.join(ROOT, "stopeps.jl_b200", "bench_states.py"))
    bs = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bs)
    from oracle.model import State
    from oracle.z2 import leg
    sites, dims, beta, log_amplitude = bs.load(name)
    L = int(round(len(sites) ** 0.5))
    grid = [[None] * L for _ in range(L)]
    for i, (a, d) in enumerate(zip(sites, dims)):
        grid[i % L][i // L] = T(np.asarray(a, float), [leg(int(p), int(q)) for p, q in d])
    return State(L, L, grid, beta, log_amplitude, "pepo")


def bench_energy_case(name, D=6, chi=36, h=3.0, state="tfim_8x8_h3_D6_chi36_beta0.4.npz"):
    """The FP64 oracle energy of a benchmark state (the stored purified 8x8
    PEPO, or state="synthetic": the seeded synthetic stand-in of the same
    shapes; D=6, chi=36 = 18+18, exact compression): the reference value of the
    benchmark's precision check."""
    if state == "synthetic":
        st = synthetic_state(8, 8, D, 0.15, 7)
        md.normalize_state(st)
    else:
        st = stored_state(state)
    m = bm.BoundaryMPS(chi, (chi // 2, chi // 2))
    en = sp.measure_energy(st, md.TFIM(1.0, h), m)
    out = dict(energy=np.array([en["energy_total"], en["energy_per_site"], en["log_norm"], en["x_sum"],
                                en["max_environment_truncation"]]), site_x=en["site_x"],
               state=state)
    np.savez_compressed(os.path.join(HERE, name), **out)
    print(name, "E", en["energy_per_site"], flush=True)


def config1_case(name, Ns=4):
    """The plain-method configuration end to end (4x4, D=4 = 2+2, chi=16 = 8+8,
    h=0.7, tau=0.05, beta0=0.5, seed 1) with Ns draws evolved to beta=1 and
    measured at 0.5 and 1: purification, draws, grouping, full-update evolution,
    weights and the ensemble curve."""
    c = dr.RunConfig(Lx=4, Ly=4, J=1.0, h=0.7, beta0=0.5, beta_log=[1.0], beta_measure=[0.5, 1.0],
                     delta_tau_pur=0.05, delta_tau_peps=0.05, D_pur=4, D_peps=4, bond_space_pur=(2, 2),
                     bond_space_peps=(2, 2), chi_environment=16, environment_space=(8, 8), Ns=Ns, seed=1)
    st, rows = dr.run_purification(c)
    res = dr.run_stochastic(c, st)
    curve = res["curve"]
    out = dict(pur_lnZ=np.array([r["lnZ"] for r in rows]), pur_energy=np.array([r["energy_per_site"] for r in rows]),
               beta=np.array([r["beta"] for r in curve]), energy=np.array([r["energy_per_site"] for r in curve]),
               lnZ=np.array([r["lnZ"] for r in curve]), eta=np.array([r["eta"] for r in curve]),
               magnetization=np.array([r.get("magnetization", np.nan) for r in curve]),
               draw_logp=np.array([d["log_probability"] for d in res["draws"]]),
               draw_cfg=np.stack([np.asarray(d["configuration"]) for d in res["draws"]]),
               multiplicity=np.asarray(res["grouping"]["multiplicity"]))
    np.savez_compressed(os.path.join(HERE, name), **out)
    print(name, out["energy"], out["lnZ"], out["eta"], flush=True)


def pipeline_case(name):
    c = dr.RunConfig(Lx=2, Ly=2, J=1.0, h=0.7, beta0=0.2, beta_log=[0.1, 0.2, 0.3], beta_measure=[0.2, 0.3],
                     delta_tau_pur=0.05, delta_tau_peps=0.05, D_pur=2, D_peps=2, bond_space_pur=(1, 1),
                     bond_space_peps=(1, 1), chi_environment=4, environment_space=(2, 2), Ns=6, seed=3)
    st, rows = dr.run_purification(c)
    res = dr.run_stochastic(c, st)
    curve = res["curve"]
    out = dict(pur_beta=np.array([r["beta"] for r in rows]), pur_lnZ=np.array([r["lnZ"] for r in rows]),
               pur_energy=np.array([r["energy_per_site"] for r in rows]),
               beta=np.array([r["beta"] for r in curve]), energy=np.array([r["energy_per_site"] for r in curve]),
               energy_error=np.array([r["energy_per_site_error"] for r in curve]),
               lnZ=np.array([r["lnZ"] for r in curve]), eta=np.array([r["eta"] for r in curve]),
               draw_logp=np.array([d["log_probability"] for d in res["draws"]]),
               draw_cfg=np.stack([np.asarray(d["configuration"]) for d in res["draws"]]),
               multiplicity=np.asarray(res["grouping"]["multiplicity"]),
               log_weights=np.array([[s["log_weight"] for s in node] for node in res["samples"]]))
    np.savez_compressed(os.path.join(HERE, name), **out)
    print(name, out["energy"], out["lnZ"])


if __name__ == "__main__":
    only = sys.argv[1:]
    if only:
        for name in only:
            {"pepo_4x4_D4.npz": lambda: pepo_case("pepo_4x4_D4.npz", 4, 4, 0.7, 4, (2, 2), 16, (8, 8), 0.5, 0.05,
                                                  [(16, (8, 8)), (24, (12, 12))], peps_D=4, peps_space=(2, 2),
                                                  peps_chi=16, peps_env_space=(8, 8), ndraws=4, seed=1),
             "headline_4x4_D6_chi36.npz": lambda: headline_case("headline_4x4_D6_chi36.npz"),
             "bench_8x8_D6_chi36_energy.npz": lambda: bench_energy_case("bench_8x8_D6_chi36_energy.npz"),
             "config1_4x4_D4_run.npz": lambda: config1_case("config1_4x4_D4_run.npz"),
             "bench_8x8_D6_chi36_synthetic_energy.npz":
                 lambda: bench_energy_case("bench_8x8_D6_chi36_synthetic_energy.npz", state="synthetic")}[name]()
        sys.exit(0)
    # 3x3, D=4 PEPO; boundary chi 8 truncates, 16 is exact; PEPS step at D=2 exercises the ALS
    pepo_case("pepo_3x3_D4.npz", 3, 3, 0.7, 4, (2, 2), 16, (8, 8), 0.2, 0.05,
              [(8, (4, 4)), (16, (8, 8))], peps_D=2, peps_space=(1, 1), peps_chi=8, peps_env_space=(4, 4))
    # 2x3 strong field, small D and chi everywhere (truncating boundaries and bonds)
    pepo_case("pepo_2x3_D2.npz", 2, 3, 3.0, 2, None, 6, None, 0.3, 0.05, [(4, None), (6, None)],
              peps_D=2, peps_space=None, peps_chi=4, peps_env_space=None, ndraws=6, seed=5,
              update=fu.FullUpdate(max_iterations=8, linear_max_iterations=40))
    pipeline_case("pipeline_2x2.npz")
    # the plain-method config (4x4, D=4, chi=16, h=0.7, beta0=0.5, tau=0.05): large enough
    # for the multi-CTA QR (chi=16) and Jacobi SVD (chi=24) paths of the engine
    pepo_case("pepo_4x4_D4.npz", 4, 4, 0.7, 4, (2, 2), 16, (8, 8), 0.5, 0.05,
              [(16, (8, 8)), (24, (12, 12))], peps_D=4, peps_space=(2, 2), peps_chi=16, peps_env_space=(8, 8),
              ndraws=4, seed=1)
    # the headline shapes (D=6, chi=36 = 18+18, h=3.0, tau=0.02) on 4x4, synthetic seeded PEPO
    headline_case("headline_4x4_D6_chi36.npz")
    # the benchmark's precision reference: the 8x8 beta0 state's FP64 energy
    bench_energy_case("bench_8x8_D6_chi36_energy.npz")
    bench_energy_case("bench_8x8_D6_chi36_synthetic_energy.npz", state="synthetic")
    # the plain-method configuration end to end with four draws evolved to beta = 1
    config1_case("config1_4x4_D4_run.npz")
