"""The sharded ensemble driver on world-size-2 gloo (CPU), against the serial run.

The numerical operations are supplied by the CPU oracle through the drivers'
ops interface, so this tests the host-side distribution logic of
``run_stochastic`` (round-robin draws, representative owners, record
gathers, collective error propagation) without a GPU.
"""
import datetime
import math
import multiprocessing as mp
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


class OracleOps:
    """The drivers' ops on the CPU oracle (test-only)."""

    def __init__(self, c):
        from oracle import boundary as bm, full_update as fu, model as md
        self.c = c
        self.bm, self.fu, self.md = bm, fu, md

    def _m(self, m):
        from oracle import diagonal as dg
        sp = None if m.sector_space is None else (m.sector_space.n0, m.sector_space.n1)
        if type(m).__name__ == "BoundaryMPSDiagonal":
            return dg.BoundaryMPSDiagonal(m.chi, sp)
        if type(m).__name__ == "BoundaryMPSRowVariational":
            from oracle import variational as va
            return va.BoundaryMPSRowVariational(m.chi, sp, m.max_sweep, m.threshold_sweep)
        if type(m).__name__ == "BoundaryMPSDiagonalVariational":
            from oracle import diagonal_variational as dv
            return dv.BoundaryMPSDiagonalVariational(m.chi, sp, m.max_sweep, m.threshold_sweep)
        return self.bm.BoundaryMPS(m.chi, sp)

    @staticmethod
    def _sampler(cache):
        from oracle import diagonal as dg, sampling as sp
        return dg if isinstance(cache, dg.DiagonalSamplingCache) else sp

    def identity(self):
        st = self.md.identity_pepo(self.c.lattice.Lx, self.c.lattice.Ly)
        rec = self.md.normalize_state(st)
        return st, [v for _, v in rec]

    def sampling_cache(self, state, method, kind="auxiliary"):
        from oracle import diagonal as dg, sampling as sp
        from oracle import diagonal_variational as dv
        m = self._m(method)
        if isinstance(m, (dg.BoundaryMPSDiagonal, dv.BoundaryMPSDiagonalVariational)):
            return dg.DiagonalSamplingCache(state, m, kind=kind)
        return sp.SamplingCache(state, m, kind=kind)

    @staticmethod
    def _repairs(d):
        reps = d.get("repairs", [])
        neg = [r for r in reps if "minimum_relative_eigenvalue" in r]
        return dict(metric_repairs=sum(1 for r in neg if r["negative_eigenvalues"] > 0),
                    zero_proposals=sum(1 for r in reps if r.get("reason") == "zero_proposal_weights"),
                    min_relative_eigenvalue=min([0.0] + [r["minimum_relative_eigenvalue"] for r in neg]))

    def sample(self, cache, uniforms):
        d = self._sampler(cache).sample_configuration(cache, uniforms=uniforms)
        return dict(configuration=np.asarray(d["configuration"]), log_probability=d["log_probability"],
                    max_environment_truncation=d["max_environment_truncation"], **self._repairs(d))

    def export_state(self, state):
        from oracle import z2
        Lx, Ly = state.Lx, state.Ly
        sites = [state[x, y] for y in range(Ly) for x in range(Lx)]
        dims = [[(int(np.sum(p == 0)), int(np.sum(p == 1))) for p in A.p] for A in sites]
        return dict(sites=[A.a.copy() for A in sites], dims=np.asarray(dims), is_pepo=state.kind == "pepo",
                    beta=state.beta, log_amplitude=state.log_amplitude)

    def _state(self, blob, Lx, Ly):
        from oracle.model import State
        from oracle.z2 import T, leg
        grid = [[None] * Ly for _ in range(Lx)]
        for i, (a, ld) in enumerate(zip(blob["sites"], blob["dims"])):
            grid[i % Lx][i // Lx] = T(np.asarray(a, float), [leg(int(p), int(q)) for p, q in ld])
        return State(Lx, Ly, grid, float(blob["beta"]), float(blob["log_amplitude"]),
                     "pepo" if blob["is_pepo"] else "peps")

    def import_state(self, blob, like):
        return self._state(blob, like.Lx, like.Ly)

    def state_from(self, blob, c):
        return self._state(blob, c.lattice.Lx, c.lattice.Ly)

    def probability(self, cache, configuration):
        d = self._sampler(cache).sample_configuration(cache, configuration=np.asarray(configuration).tolist())
        return dict(log_probability=d["log_probability"],
                    max_environment_truncation=d["max_environment_truncation"], **self._repairs(d))

    def project(self, state, configuration):
        from oracle import sampling as sp
        st, rec = sp.project_configuration(state, np.asarray(configuration).tolist())
        return st, [v for _, v in rec]

    def measure_energy(self, state, method):
        from oracle import diagonal as dg, sampling as sp
        from oracle import diagonal_variational as dv
        m = self._m(method)
        mod = dg if isinstance(m, (dg.BoundaryMPSDiagonal, dv.BoundaryMPSDiagonalVariational)) else sp
        return dict(mod.measure_energy(state, self.md.TFIM(self.c.model.J, self.c.model.h, self.c.model.fields), m))

    def lognorm(self, state, method):
        from oracle import diagonal as dg
        from oracle import diagonal_variational as dv
        m = self._m(method)
        diag = isinstance(m, (dg.BoundaryMPSDiagonal, dv.BoundaryMPSDiagonalVariational))
        return dict((dg if diag else self.bm).lognorm(state, m))

    def evolution_step(self, state, delta, D, method, space):
        u = self.c.update
        opts = self.fu.FullUpdate(u.max_iterations, u.error_tolerance, u.diagonal_shift,
                                  u.linear_max_iterations, u.linear_tolerance)
        r = self.fu.evolution_step(state, self.md.TFIM(self.c.model.J, self.c.model.h, self.c.model.fields), delta, D, opts,
                                   self._m(method), order=self.c.trotter_order,
                                   space=None if space is None else (space.n0, space.n1),
                                   record_entropy=self.c.record_boundary_entropy)
        return dict(r, log_normalization_sum=sum(v for _, v in r["normalizations"]))


def _config(sps):
    return sps.RunConfig(lattice=sps.Lattice(2, 2), model=sps.TFIM(1.0, 0.7), beta0=0.1, beta_log=[0.1, 0.2],
                         beta_measure=[0.1, 0.2], delta_tau_pur=0.05, delta_tau_peps=0.05, D_pur=2, D_peps=2,
                         chi_environment=4, Ns=5, seed=9, resampling=sps.ResamplingOptions(enabled=False))


def _config_resampling(sps):
    """An event at beta = 0.3 (eta_th = 1) with two sweeps, Ns = 6."""
    return sps.RunConfig(lattice=sps.Lattice(2, 2), model=sps.TFIM(1.0, 0.7), beta0=0.1, beta_log=[0.1, 0.3],
                         beta_measure=[0.1, 0.3], delta_tau_pur=0.05, delta_tau_peps=0.05, D_pur=2, D_peps=2,
                         chi_environment=4, Ns=6, seed=5,
                         resampling=sps.ResamplingOptions(enabled=True, eta_th=1.0, max_resample_sweep=2))


def _run(sps, execution=None, fail_rank=None, resampling=False):
    c = _config_resampling(sps) if resampling else _config(sps)
    ops = OracleOps(c)
    if fail_rank is not None and execution is not None and execution.rank() == fail_rank:
        def bad(*a, **k):
            raise RuntimeError("planted failure")
        ops.sample = bad
    cp = sps.run_purification(c, ops=ops, identity=ops.identity)
    return sps.run_stochastic(c, cp, execution=execution, ops=ops)


def _worker(rank, world, port, q, fail_rank, resampling=False):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        import __graft_entry__ as ge
        sps = ge.load_package()
        try:
            res = _run(sps, sps.TorchExecution(), fail_rank, resampling)
            out = None if res is None else [(r["beta"], r["energy_per_site"], r["lnZ"], r["eta"])
                                             for r in res["observables"]["curve"]]
            events = None if res is None else _event_summary(res)
            q.put((rank, "ok", out, None if res is None else res["metadata"]["mpi_size"], events))
        except RuntimeError as ex:
            q.put((rank, "error", str(ex), None, None))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _event_summary(res):
    """Members, fresh draws, selected representatives and weights of each resampling event."""
    out = []
    for ev in res["diagnostics"]["events"]:
        out.append(dict(members=[s["members"] for s in ev["sweeps"]],
                        draws=[[(d["index"], tuple(np.asarray(d["configuration"]).reshape(-1).tolist()),
                                 d["log_probability"]) for d in s["draws"]] for s in ev["sweeps"]],
                        post=[(r["id"], r["count"], r["relative_log_weight"], r["weight_log_scale"])
                              for r in ev["post"]],
                        stop=ev["stop_reason"],
                        moved=sum(1 for r in ev["post"]
                                  if {q["id"]: q["owner"] for q in ev["pre"] + ev["fresh"]}[r["id"]] != r["owner"])))
    return out


def _spawn(world, fail_rank=None, resampling=False):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, fail_rank, resampling)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=600) for _ in procs]
    for p in procs:
        p.join(timeout=120)
    return sorted(results)


def test_two_ranks_match_serial(sps):
    serial = _run(sps)
    ref = [(r["beta"], r["energy_per_site"], r["lnZ"], r["eta"]) for r in serial["observables"]["curve"]]
    results = _spawn(2)
    assert [r[1] for r in results] == ["ok", "ok"]
    rank0 = results[0]
    assert rank0[3] == 2 and results[1][2] is None      # rank 0 returns the record, rank 1 nothing
    for a, b in zip(rank0[2], ref):
        for x, y in zip(a, b):
            assert (math.isnan(x) and math.isnan(y)) or abs(x - y) <= 1e-12 * max(1.0, abs(y))


def test_failure_on_one_rank_raises_on_all(sps):
    results = _spawn(2, fail_rank=1)
    assert [r[1] for r in results] == ["error", "error"]
    assert all("planted failure" in r[2] for r in results)


class BatchedOracleOps(OracleOps):
    """The drivers' batched ops (sample/project/measure/lognorm/evolution
    batches), each a loop over the single oracle operation: exercises the
    batched code path of run_stochastic on the CPU."""

    def __init__(self, c):
        super().__init__(c)
        self.calls = {}

    def _count(self, name, n):
        self.calls[name] = self.calls.get(name, 0) + 1
        assert n >= 1

    def sample_batch(self, cache, uniforms):
        self._count("sample_batch", len(uniforms))
        return [self.sample(cache, u) for u in uniforms]

    def project_batch(self, state, configurations):
        self._count("project_batch", len(configurations))
        return [self.project(state, c) for c in configurations]

    def measure_energy_batch(self, states, method):
        self._count("measure_energy_batch", len(states))
        return [self.measure_energy(s, method) for s in states]

    def lognorm_batch(self, states, method):
        self._count("lognorm_batch", len(states))
        return [self.lognorm(s, method) for s in states]

    def evolution_step_batch(self, states, deltas, D, method, space):
        self._count("evolution_step_batch", len(states))
        return [self.evolution_step(s, d, D, method, space) for s, d in zip(states, deltas)]


def test_batched_ops_match_single_ops(sps):
    """run_stochastic through the batched ops: one call per phase (draws,
    projections, observations, each evolution step), same result as the
    single-operation path."""
    serial = _run(sps)
    c = _config(sps)
    ops = BatchedOracleOps(c)
    cp = sps.run_purification(c, ops=ops, identity=ops.identity)
    res = sps.run_stochastic(c, cp, ops=ops)
    assert ops.calls["sample_batch"] == 1
    assert ops.calls["project_batch"] == 1
    assert ops.calls["evolution_step_batch"] >= 1
    for a, b in zip(res["observables"]["curve"], serial["observables"]["curve"]):
        for k in ("beta", "energy_per_site", "lnZ", "eta"):
            x, y = a[k], b[k]
            assert (math.isnan(x) and math.isnan(y)) or abs(x - y) <= 1e-12 * max(1.0, abs(y))
    assert [d["configuration"].tolist() for d in res["diagnostics"]["born_draws"]] == \
        [d["configuration"].tolist() for d in serial["diagnostics"]["born_draws"]]


def test_two_ranks_resampling_match_serial(sps):
    """An annealed resampling event over two gloo ranks (scores and draws on
    their owners, fresh samples by representative owner, selected particles
    moved to their new ranks) gives the serial run's members, draws, selected
    representatives with their weights, and curve."""
    serial = _run(sps, resampling=True)
    ref = [(r["beta"], r["energy_per_site"], r["lnZ"], r["eta"]) for r in serial["observables"]["curve"]]
    ref_events = _event_summary(serial)
    assert ref_events
    results = _spawn(2, resampling=True)
    assert [r[1] for r in results] == ["ok", "ok"], results
    rank0 = results[0]
    for a, b in zip(rank0[2], ref):
        for x, y in zip(a, b):
            assert (math.isnan(x) and math.isnan(y)) or abs(x - y) <= 1e-12 * max(1.0, abs(y))
    for ev, rv in zip(rank0[4], ref_events):
        assert ev["members"] == rv["members"] and ev["stop"] == rv["stop"]
        for s1, s2 in zip(ev["draws"], rv["draws"]):
            assert [d[:2] for d in s1] == [d[:2] for d in s2]
            for d1, d2 in zip(s1, s2):
                assert abs(d1[2] - d2[2]) <= 1e-12 * max(1.0, abs(d2[2]))
        assert [p[:2] for p in ev["post"]] == [p[:2] for p in rv["post"]]
        assert ev["moved"] > 0 and rv["moved"] == 0   # particles changed ranks on two, none on one
        for p1, p2 in zip(ev["post"], rv["post"]):
            assert abs(p1[2] - p2[2]) <= 1e-12 and abs(p1[3] - p2[3]) <= 1e-12 * max(1.0, abs(p2[3]))


def test_host_driver_with_site_fields(sps):
    """The host driver carries per-site fields to the contraction ops: the
    purification records equal the oracle driver's own run of the same model."""
    from oracle import driver as odr
    f = (0.5, 0.9, 0.7, 1.1)
    c = sps.RunConfig(lattice=sps.Lattice(2, 2), model=sps.TFIM(1.0, 0.7, fields=f), beta0=0.1, beta_log=[0.1],
                      beta_measure=[0.1], delta_tau_pur=0.05, delta_tau_peps=0.05, D_pur=2, D_peps=2,
                      chi_environment=4, Ns=2, seed=9, resampling=sps.ResamplingOptions(enabled=False))
    ops = OracleOps(c)
    cp = sps.run_purification(c, ops=ops, identity=ops.identity)
    _, rows = odr.run_purification(odr.RunConfig(Lx=2, Ly=2, J=1.0, h=0.7, fields=f, beta0=0.1, beta_log=[0.1],
                                                 beta_measure=[0.1], delta_tau_pur=0.05, D_pur=2, D_peps=2,
                                                 chi_environment=4, Ns=2, seed=9))
    for a, b in zip(cp.purification, rows):
        for k in ("lnZ", "energy_per_site"):
            assert (math.isnan(a[k]) and math.isnan(b[k])) or abs(a[k] - b[k]) <= 1e-12 * max(1.0, abs(b[k]))
    uniform = sps.run_purification(c.__class__(**{**c.__dict__, "model": sps.TFIM(1.0, 0.7)}), ops=OracleOps(
        c.__class__(**{**c.__dict__, "model": sps.TFIM(1.0, 0.7)})), identity=ops.identity)
    assert abs(uniform.purification[-1]["lnZ"] - cp.purification[-1]["lnZ"]) > 1e-6   # the fields matter


def test_host_driver_with_diagonal_contraction(sps):
    """``RunConfig(contraction=BoundaryMPSDiagonal)`` through the host driver:
    purification records, draws and the sampled curve equal the oracle
    driver's own run on diagonal boundaries (draws consume their uniforms in
    the anti-diagonal order, the parameter record names the method)."""
    from oracle import driver as dr
    kw = dict(beta0=0.1, beta_log=[0.1, 0.2], beta_measure=[0.1, 0.2], delta_tau_pur=0.05, delta_tau_peps=0.05,
              D_pur=2, D_peps=2, chi_environment=4, Ns=3, seed=9)
    c = sps.RunConfig(lattice=sps.Lattice(2, 3), model=sps.TFIM(1.0, 0.7), contraction=sps.BoundaryMPSDiagonal,
                      resampling=sps.ResamplingOptions(enabled=False), **kw)
    sps.validate_config(c)
    ops = OracleOps(c)
    cp = sps.run_purification(c, ops=ops, identity=ops.identity)
    oc = dr.RunConfig(Lx=2, Ly=3, J=1.0, h=0.7, diagonal=True, **{k: v for k, v in kw.items()})
    _, rows = dr.run_purification(oc)
    for a, b in zip(cp.purification, rows):
        for k in ("lnZ", "energy_per_site"):
            assert (math.isnan(a[k]) and math.isnan(b[k])) or abs(a[k] - b[k]) <= 1e-12 * max(1.0, abs(b[k]))
    res = sps.run_stochastic(c, cp, ops=ops)
    draws = res["diagnostics"]["born_draws"]
    assert len(draws) == 3 and all(np.isfinite(d["log_probability"]) for d in draws)
    p = sps.parameter_dict(c)
    assert p["contraction"] == "BoundaryMPS-Diagonal"
    assert p["sampling_site_order"][:3] == [(1, 1), (2, 1), (1, 2)]


def test_host_driver_with_row_variational_contraction(sps):
    """``RunConfig(contraction=BoundaryMPSRowVariational)`` through the host
    driver equals the oracle's exact-compression run at a chi above every bond
    (the variational fit is then exact) and names the method in its record."""
    from oracle import driver as dr
    kw = dict(beta0=0.1, beta_log=[0.1, 0.2], beta_measure=[0.1, 0.2], delta_tau_pur=0.05, delta_tau_peps=0.05,
              D_pur=2, D_peps=2, chi_environment=64, Ns=3, seed=9)
    c = sps.RunConfig(lattice=sps.Lattice(3, 2), model=sps.TFIM(1.0, 0.7),
                      contraction=sps.BoundaryMPSRowVariational, resampling=sps.ResamplingOptions(enabled=False),
                      **kw)
    sps.validate_config(c)
    ops = OracleOps(c)
    cp = sps.run_purification(c, ops=ops, identity=ops.identity)
    _, rows = dr.run_purification(dr.RunConfig(Lx=3, Ly=2, J=1.0, h=0.7, **kw))
    for a, b in zip(cp.purification, rows):
        for k in ("lnZ", "energy_per_site"):
            assert (math.isnan(a[k]) and math.isnan(b[k])) or abs(a[k] - b[k]) <= 1e-11 * max(1.0, abs(b[k]))
    assert sps.parameter_dict(c)["contraction"] == "BoundaryMPS-Row-Variational"
    cd = sps.RunConfig(lattice=sps.Lattice(3, 2), model=sps.TFIM(1.0, 0.7),
                       contraction=sps.BoundaryMPSDiagonalVariational, resampling=sps.ResamplingOptions(enabled=False),
                       **kw)
    sps.validate_config(cd)
    ops = OracleOps(cd)
    cpd = sps.run_purification(cd, ops=ops, identity=ops.identity)
    for a, b in zip(cpd.purification, rows):
        for k in ("lnZ", "energy_per_site"):
            assert (math.isnan(a[k]) and math.isnan(b[k])) or abs(a[k] - b[k]) <= 1e-11 * max(1.0, abs(b[k]))
    p = sps.parameter_dict(cd)
    assert p["contraction"] == "BoundaryMPS-Diagonal-Variational" and p["sampling_site_order"][1] == (2, 1)
