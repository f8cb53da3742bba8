#!/usr/bin/env python
"""Born samples/s on the 8x8 open TFIM (J=1, h=3.0), D=6 (3+3), chi=36 (18+18).

One step = W perfect Born draws (``sample_configuration``, src/sampling/born.jl:86-163)
drawn at the same time from a device-resident SamplingCache of the purified
beta0 = 0.4 PEPO (stored, bench_states.py): per draw eight row absorptions and
64 conditionals.  The headline `value` is the zip-up absorption path
(FP64); the plain FP64 path (the reference's exact LQ + truncated-SVD
compression, one sample per launch sequence) draws the same sample ids beside
it (`plain_fp64`, `agreement_vs_plain`).  `pipeline` times the rest of the
per-sample unit on the same PEPO: projection, one full-update Trotter step
(src/evolution/full_update.jl:559-597) and one energy measurement
(src/measurement/energy.jl:31-78), and composes the per-sample rate for
beta 0.4 -> 2.0 at tau = 0.02.  Every rank draws its own samples (weak
scaling: samples shard with no data-path collective); rank 0 prints one JSON
line.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--concurrency C]
  python bench.py --probe NAME [ARGS]   # one hot operation, for profiling (see PROBES)
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

LX = LY = 8
D = 6
CHI = 36
H_FIELD = 3.0
SEED = 1
PEPO_EPS = 0.15
PEPO_SEED = 7
BETA0, BETA_MAX, DTAU = 0.4, 2.0, 0.02
MEASURE_BETAS = [0.5 + 0.25 * k for k in range(7)]   # 0.5, 0.75, ..., 2.0
METRIC = "Born samples/s at 8x8 D6 χ36: batched mixed-prec vs plain FP64 GPU, ΔE≤1e-4"
ORACLE_ENERGY = os.path.join(ROOT, "tests", "golden", "bench_8x8_D6_chi36_energy.npz")

PROBES = """probes (one hot operation on a representative input, run once to warm up and once more):
  svd_left          U-only Jacobi of a 648x648 LQ-preconditioned block
  tcgemm [mode m n k] the tcgen05 contraction GEMM (tf32 | 3xtf32 | 3xbf16), default 3xtf32 8192^3
  qr                blocked Householder QR of a 23328x648 block
  topk [W] [gram]   leading 18 triplets of a 648x648 graded block (1/W of the SMs)
  gemm              FP64 GEMM 23328x648x648 and the 648x648x23328 Gram
  draw [synthetic]  one Born draw, 8x8 D=6 chi=36, exact compression (purified beta0 PEPO, or the
                    seeded synthetic stand-in of the same shapes)
  zipdraw [synthetic] the same draw with the zip-up absorption
  scale             zip-up draws at 12x12 D=8 chi=64 (32+32): 1 and 4 at a time
  fustep [L]        one full-update Trotter step + energy, L x L D=6 chi=36 (default 8): both absorptions,
                    FP64 and 3xTF32 contractions
  purify [L] [s] [p] purification of the L x L TFIM to beta0 = 0.4 at D=6 chi=36 within s seconds
                    (precision p), the state saved under --out
  adjoint [L] [D] [chi] lognorm and its reverse-mode derivative (row checkpoints; the full tape where it
                    fits in 60 GB) and the per-site field derivatives, on the seeded synthetic L x L PEPO
                    (default 8, D=6, chi=36)"""


def parse():
    p = argparse.ArgumentParser(epilog=PROBES, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=4)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--concurrency", type=int, default=8,
                   help="samples drawn at the same time on one GPU (own stream and workspace each)")
    p.add_argument("--no-pipeline", action="store_true", help="skip the full-update / measurement sub-lines")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    p.add_argument("--probe", nargs="+", metavar="NAME", help="run one probe instead of the benchmark")
    p.add_argument("--out", default="probe_out", help="directory for files a probe writes")
    return p.parse_args()


def workload_config(extra=None):
    c = {"workload": "tfim_8x8_D6_chi36_born_draw", "Lx": LX, "Ly": LY, "J": 1.0, "h": H_FIELD, "D": D,
         "bond_space": [D // 2, D // 2], "chi_sampling": CHI, "sampling_space": [CHI // 2, CHI // 2],
         "pepo": "the purified beta0 = 0.4 PEPO of the 8x8 TFIM (10 full-update steps at tau = 0.02 from the "
                 "identity, D=6, chi=36; stored in stopeps.jl_b200/states/)",
         "step": "W Born draws from a device-resident SamplingCache",
         "uniforms": "numpy default_rng([seed, sample_id])", "seed": SEED,
         "l2": "inputs larger than L2 (the south boundaries and candidate double layers of the cache, ~0.6 GB)"}
    if extra:
        c.update(extra)
    return c


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU reference algorithm (the oracle restatement), drawn row by row
# ---------------------------------------------------------------------------
class OracleRowDraws:
    """Reference-algorithm Born draws on the CPU oracle with real boundaries.

    The SamplingCache (PEPO double layers, candidates, the Ly south boundaries
    by the exact compression) is built once, untimed, as the reference builds
    it once per checkpoint (born.jl:56-73).  ``step()`` then advances the
    current draw by one row (its Lx conditionals and the north absorption);
    after Ly rows the next sample id starts, so consecutive steps are whole
    draws of sample ids 1, 2, ..."""

    def __init__(self):
        import numpy as np
        from oracle import boundary as bm, model as omd, sampling as osp
        from oracle.z2 import T, leg
        import __graft_entry__ as ge
        sites, dims, beta, log_amplitude = ge.load_package().bench_states.load()
        grid = [[None] * LY for _ in range(LX)]
        for i, (a, ld) in enumerate(zip(sites, dims)):
            grid[i % LX][i // LX] = T(np.asarray(a, float), [leg(int(p), int(q)) for p, q in ld])
        st = omd.State(LX, LY, grid, beta, log_amplitude, "pepo")
        self.osp = osp
        self.ge = ge
        t = time.perf_counter()
        self.cache = osp.SamplingCache(st, bm.BoundaryMPS(CHI, (CHI // 2, CHI // 2)))
        self.setup_s = time.perf_counter() - t
        self.sample_id = 0
        self.rows = None
        self.draws = []

    def step(self):
        if self.rows is None:
            self.sample_id += 1
            u = self.ge.load_package().sample_uniforms(SEED, self.sample_id, LX * LY)
            self.rows = self.osp.sample_rows(self.cache, uniforms=u)
        try:
            next(self.rows)
        except StopIteration as done:
            self.draws.append((self.sample_id, done.value))
            self.rows = None
            self.step()


def reference_arm(args, rank, world):
    """The reference algorithm on the host cores (the Julia reference itself cannot
    run here: no Julia).  A step is one row of a real draw (see OracleRowDraws);
    value = (rows timed / Ly) draws over the timed seconds."""
    if rank != 0:
        return
    cores = os.cpu_count()
    rd = OracleRowDraws()
    for _ in range(args.warmup):
        rd.step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        rd.step()
    dt = time.perf_counter() - t0
    value = (args.steps / LY) / dt
    sample = (f"{args.steps} consecutive rows of real draws (sample ids from 1; {args.steps / LY:.2f} draws; a row is "
              f"{LX} conditionals + the north absorption), after {args.warmup} warm-up rows; the SamplingCache "
              f"(7 south absorptions) built untimed in {rd.setup_s:.1f} s; CPU oracle (NumPy/OpenBLAS FP64, "
              f"{cores} threads) restating the reference algorithm (exact LQ + truncated SVD), which cannot run "
              "here as Julia is not installed")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (a TFIM state prepared by this engine, stored; no dataset)", "config": workload_config({"step": "one row of a Born draw (reference arm)"}),
            "cpu_baseline": {"value": value, "unit": "samples/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline_sample(rows=2):
    """The oracle's reference algorithm on `rows` rows of a real draw (cache built untimed)."""
    rd = OracleRowDraws()
    t0 = time.perf_counter()
    for _ in range(rows):
        rd.step()
    dt = time.perf_counter() - t0
    return {"value": (rows / LY) / dt, "unit": "samples/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"the first {rows} rows of real draw 1 ({dt:.1f} s; {LX} conditionals + north absorption "
                      f"each; SamplingCache built untimed in {rd.setup_s:.1f} s), scaled to a draw of {LY} rows; "
                      "CPU oracle (NumPy/OpenBLAS FP64), reference algorithm"}


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
def purified_state(sps, e):
    """The stored beta0 = 0.4 PEPO of the 8x8 TFIM (bench_states.py) on the engine."""
    sites, dims, beta, log_amplitude = sps.bench_states.load()
    return e.upload_state(sites, dims, True, beta=beta, log_amplitude=log_amplitude)


def measure_fp64_peak(torch, device):
    """cuBLAS DGEMM 8192^3 through torch (the FP64 denominator of the roofline)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    best = 0.0
    for _ in range(4):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def roofline_of(stats, peak, note):
    """The dominant FLOP-counted kernel of a per-kernel profile against the FP64 peak."""
    tot = sum(v["ms"] for k, v in stats.items() if "." not in k and not k.startswith("gemm_gather "))
    cands = [(k, v) for k, v in stats.items() if v["flops"] > 0 and "." not in k and not k.startswith("gemm_gather ")]
    name, v = max(cands, key=lambda kv: kv[1]["ms"])
    per_launch_flops = v["flops"] / v["count"]
    avg_ms = v["ms"] / v["count"]
    achieved = per_launch_flops / (avg_ms * 1e-3) / 1e12
    return {"bound": "tensor", "kernel": name, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak, "traffic": None, "note": note,
            "peak_source": "FP64: cuBLAS DGEMM 8192^3 measured in this run (FP64 is not in MEASURED_PEAKS.json); "
                           "tensor-core FP64 and DFMA share the FP64 rate on B200",
            "share_of_profiled_time": v["ms"] / tot if tot else None,
            "kernels": {k: {"ms": round(s["ms"], 3), "count": s["count"],
                            "share": round(s["ms"] / tot, 4) if tot and "." not in k else None,
                            "tflops": round(s["flops"] / (s["ms"] * 1e-3) / 1e12, 3)
                            if s["ms"] > 0 and s["flops"] > 0 else None}
                        for k, s in sorted(stats.items(), key=lambda kv: -kv[1]["ms"])
                        if not k.startswith("gemm_gather ")}}


def ours_arm(args, rank, world, local_rank):
    import numpy as np
    import torch
    import __graft_entry__ as ge
    sps = ge.load_package()
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local_rank)
    e = sps.Engine(LX, LY, sps.TFIM(1.0, H_FIELD), device=local_rank)
    st = purified_state(sps, e)
    space = sps.Z2Space(CHI // 2, CHI // 2)
    W = max(1, args.concurrency)
    L = LX * LY

    # sample ids: rank r of N draws ids r+1, r+1+N, ...; warm-up, timed and end-to-end draws use disjoint ids
    def ids_of(first_step, nsteps):
        out = []
        for s in range(first_step, first_step + nsteps):
            out.append([1 + rank + world * (s * W + j) for j in range(W)])
        return out

    warm_ids = ids_of(0, args.warmup)
    timed_ids = ids_of(args.warmup, args.steps)
    e2e_ids = ids_of(args.warmup + args.steps, args.steps)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def draw(cache, ids):
        if len(ids) == 1:
            d = sps.sample_configuration(cache, uniforms=sps.sample_uniforms(SEED, ids[0], L))
            return [dict(d, uid=ids[0])]
        u = np.stack([sps.sample_uniforms(SEED, k, L) for k in ids])
        cfg, lp = sps.sample_batch(cache, u)
        return [{"configuration": c, "log_probability": l, "uid": k} for c, l, k in zip(cfg, lp, ids)]

    def measure(cache, batch_ids, warm, e2e=None, concurrency=1):
        """Device-timed draws of the id batches in `batch_ids` (one step each); `e2e`
        batches are drawn again through the public API and timed by the wall clock."""
        e.set_concurrency(concurrency)
        for ids in warm:
            draw(cache, ids)
        barrier()
        n0, _ = e.counters()
        draws = []
        with Clocks(local_rank) as clk:
            e.timer_start()
            for ids in batch_ids:
                draws.extend(draw(cache, ids))
            ms = e.timer_stop()
        n1, _ = e.counters()
        barrier()
        wall = None
        if e2e:
            t0 = time.perf_counter()
            for ids in e2e:
                draw(cache, ids)
            barrier()
            wall = time.perf_counter() - t0
        t = torch.tensor([ms, wall or 0.0], dtype=torch.float64, device=f"cuda:{local_rank}")
        if dist is not None:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return {"ms": float(t[0]), "wall": float(t[1]), "launches": int(n1 - n0), "clocks": clk.summary(),
                "draws": draws}

    zcache = sps.SamplingCache(st, sps.BoundaryMPSZipUp(CHI, space))
    zip_run = measure(zcache, timed_ids, warm_ids, e2e_ids, concurrency=W)
    # the same draws with the contraction GEMMs in split TF32 on the tensor cores
    # (truncations, normalisations and log-probabilities FP64; same cache)
    e.set_precision("3xtf32")
    mixed_run = measure(zcache, timed_ids, warm_ids, e2e_ids, concurrency=W)
    e.set_precision("fp64")
    # per-kernel profile of one more batch at the same concurrency (the timed configuration; untimed)
    e.set_concurrency(W)
    e.set_profile(True)
    draw(zcache, ids_of(args.warmup + 2 * args.steps, 1)[0])
    conc_stats = e.kernel_stats()
    e.set_profile(False)
    # ... and of one serial draw (the per-kernel shares the ncu launch list is compared with)
    e.set_concurrency(1)
    e.set_profile(True)
    draw(zcache, [ids_of(args.warmup + 2 * args.steps + 1, 1)[0][0]])
    serial_stats = e.kernel_stats()
    e.set_profile(False)

    # the plain FP64 path, one sample at a time, on the first timed zip-up sample ids
    plain_steps = max(1, min(args.steps * W, 2))
    pcache = sps.SamplingCache(st, sps.BoundaryMPS(CHI, space))
    flat_timed = [k for ids in timed_ids for k in ids]
    plain_run = measure(pcache, [[k] for k in flat_timed[:plain_steps]], [[1 + rank + world * 10 ** 6]],
                        e2e=[[k] for k in flat_timed[:plain_steps]])
    del pcache
    value = world * args.steps * W / (zip_run["ms"] * 1e-3)
    e2e = world * args.steps * W / zip_run["wall"]
    mixed_value = world * args.steps * W / (mixed_run["ms"] * 1e-3)
    mmap = {d["uid"]: d for d in mixed_run["draws"]}
    msame = sum(int(np.array_equal(d["configuration"], mmap[d["uid"]]["configuration"])) for d in zip_run["draws"])
    mdlp = max(abs(d["log_probability"] - mmap[d["uid"]]["log_probability"]) for d in zip_run["draws"])
    plain_value = world * plain_steps / (plain_run["ms"] * 1e-3)
    plain_e2e = world * plain_steps / plain_run["wall"]
    zmap = {d["uid"]: d for d in zip_run["draws"]}
    same, dlp, ncmp = 0, 0.0, 0
    for dp in plain_run["draws"]:
        dz = zmap.get(dp["uid"])
        if dz is None:
            continue
        ncmp += 1
        same += int(np.array_equal(dz["configuration"], dp["configuration"]))
        dlp = max(dlp, abs(dz["log_probability"] - dp["log_probability"]))

    # precision: the beta0 state's energy per site under both absorptions against the oracle's FP64
    # value (exact compression; fixture made by tests/golden/make_golden.py)
    en_plain = sps.measure_energy(st, sps.BoundaryMPS(CHI, space))
    en_zip = sps.measure_energy(st, sps.BoundaryMPSZipUp(CHI, space))
    e.set_precision("3xtf32")
    en_mixed = sps.measure_energy(st, sps.BoundaryMPSZipUp(CHI, space))
    e.set_precision("fp64")
    oracle_e = None
    if os.path.exists(ORACLE_ENERGY):
        fx = np.load(ORACLE_ENERGY)
        if "state" in fx and str(fx["state"]) == sps.bench_states.PURIFIED_8X8:   # made for this very state
            oracle_e = float(fx["energy"][1])
    ref_e = oracle_e if oracle_e is not None else en_plain["energy_per_site"]
    precision = {"energy_per_site_oracle_fp64": oracle_e,
                 "energy_per_site_plain_fp64": en_plain["energy_per_site"],
                 "energy_per_site_zipup": en_zip["energy_per_site"],
                 "abs_delta_e_zipup_vs_oracle": abs(en_zip["energy_per_site"] - ref_e),
                 "energy_per_site_zipup_3xtf32": en_mixed["energy_per_site"],
                 "abs_delta_e_zipup_3xtf32_vs_oracle": abs(en_mixed["energy_per_site"] - ref_e),
                 "abs_delta_e_plain_vs_oracle": abs(en_plain["energy_per_site"] - ref_e),
                 "reference": "oracle" if oracle_e is not None else "plain FP64 GPU (oracle fixture missing)",
                 "tolerance": 1e-4,
                 "state": "the purified beta0 = 0.4 PEPO of the draws, chi=36 (18+18)"}

    pipeline = None
    if not args.no_pipeline:
        try:
            pipeline = pipeline_timing(sps, e, st, zip_run["draws"], W, space, np, torch, local_rank, dist)
        except Exception as ex:   # reported in the line; the draw measurement stands on its own
            e.set_concurrency(1)
            pipeline = {"error": f"{type(ex).__name__}: {ex}"}

    result = None
    if rank == 0:
        peak = measure_fp64_peak(torch, f"cuda:{local_rank}")
        roofline = roofline_of(conc_stats, peak,
                               f"per-kernel CUDA events of one batch of {W} concurrent draws (the timed "
                               "configuration: each launch's duration on its stream while the other samples' "
                               "kernels share the GPU); FLOPs counted over the nonzero Z2 blocks")
        roofline_serial = roofline_of(serial_stats, peak, "one draw alone (the ncu launch list's configuration)")
        cpu = None
        if world == 1 and not args.no_cpu:
            cpu = cpu_baseline_sample()
        n_h2d = 8 * L * W
        result = {"metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
                  "warmup": args.warmup, "ms_per_step": zip_run["ms"] / args.steps, "higher_is_better": True,
                  "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (a TFIM state prepared by this engine, stored; no dataset)",
                  "config": workload_config({"parallelism": f"samples sharded over {world} GPU(s)",
                                             "path": f"zip-up boundary absorption, FP64, {W} samples "
                                                     "concurrently (own stream and workspace each)",
                                             "samples_per_step": W}),
                  "e2e": {"value": e2e, "unit": "samples/s", "h2d_bytes_per_step": n_h2d,
                          "d2h_bytes_per_step": (4 * L + 8) * W},
                  "gpu_launches": zip_run["launches"], "clocks": zip_run["clocks"], "roofline": roofline,
                  "roofline_serial_draw": roofline_serial,
                  "cpu_baseline": cpu,
                  "plain_fp64": {"value": plain_value, "e2e": plain_e2e, "unit": "samples/s",
                                 "steps": plain_steps, "ms_per_step": plain_run["ms"] / plain_steps,
                                 "gpu_launches": plain_run["launches"], "clocks": plain_run["clocks"],
                                 "sample_ids": flat_timed[:plain_steps],
                                 "path": "reference algorithm: exact LQ sweep + truncated SVD sweep, FP64"},
                  "speedup_vs_plain_fp64": value / plain_value,
                  "mixed_3xtf32": {"value": mixed_value, "e2e": world * args.steps * W / mixed_run["wall"],
                                   "unit": "samples/s", "ms_per_step": mixed_run["ms"] / args.steps,
                                   "gpu_launches": mixed_run["launches"], "clocks": mixed_run["clocks"],
                                   "speedup_vs_plain_fp64": mixed_value / plain_value,
                                   "agreement_vs_fp64_zipup": {"draws": len(zip_run["draws"]),
                                                               "identical_configurations": msame,
                                                               "max_abs_dlogp": mdlp},
                                   "path": "zip-up absorption, contraction GEMMs 3xTF32 on tcgen05 (FP32 "
                                           "accumulation), truncations and log-weights FP64, same sample ids"},
                  "agreement_vs_plain": {"draws": ncmp, "identical_configurations": same,
                                         "max_abs_dlogp": dlp},
                  "precision": precision,
                  "pipeline": pipeline}
        print(json.dumps(result), flush=True)
    del st
    e.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def pipeline_timing(sps, e, st, draws, W, space, np, torch, local_rank, dist):
    """The rest of the per-sample unit: projection, one full-update Trotter step and one
    energy measurement of projected samples (zip-up environments, concurrency W), device-timed;
    composed with the draw rate into samples/s for beta 0.4 -> 2.0 at tau = 0.02."""
    n_steps = len(sps.step_schedule(BETA0, BETA_MAX, DTAU))
    zm = sps.BoundaryMPSZipUp(CHI, space)
    W = 1   # one sample: a full-update step at 8x8 D=6 takes tens of seconds
    cfgs = np.stack([d["configuration"] for d in draws[:W]])
    e.set_concurrency(W)
    e.timer_start()
    states, _ = sps.project_batch(st, cfgs)
    proj_ms = e.timer_stop()
    e.timer_start()
    reps = sps.evolution_step_batch(states, [DTAU] * len(states), D, zm, sps.Z2Space(D // 2, D // 2))
    fu_ms = e.timer_stop()
    e.timer_start()
    ens = sps.measure_energy_batch(states, zm)
    meas_ms = e.timer_stop()
    e.set_concurrency(1)
    n = len(states)
    per_sample_s = (fu_ms * n_steps + meas_ms * len(MEASURE_BETAS) + proj_ms) / n * 1e-3
    return {"samples": n, "concurrency": W, "environment": "zip-up boundary absorption, FP64",
            "project_ms_per_batch": proj_ms, "fu_step_ms_per_batch": fu_ms, "measure_ms_per_batch": meas_ms,
            "fu_step_ms_per_sample": fu_ms / n, "measure_ms_per_sample": meas_ms / n,
            "fu_bond_updates": reps[0]["bond_updates"], "fu_stop_reasons": {
                k: sum(r[f"stop_{k}"] for r in reps) for k in ("error_tolerance", "iteration_limit",
                                                               "residual_fallback", "disabled")},
            "energy_per_site_after_step": [r["energy_per_site"] for r in ens],
            "schedule": f"beta {BETA0} -> {BETA_MAX}, tau {DTAU}: {n_steps} steps, {len(MEASURE_BETAS)} measurements",
            "composed_seconds_per_sample": per_sample_s,
            "composed_samples_per_s_excluding_draw": 1.0 / per_sample_s if per_sample_s > 0 else None}


# ---------------------------------------------------------------------------
# probes
# ---------------------------------------------------------------------------
def graded(m, n, decay, seed):
    import numpy as np
    rng = np.random.default_rng(seed)
    u, _ = np.linalg.qr(rng.standard_normal((m, min(m, n))))
    v, _ = np.linalg.qr(rng.standard_normal((n, min(m, n))))
    return (u * np.exp(-decay * np.arange(min(m, n)))) @ v.T


def probe(argv, out="probe_out"):
    import numpy as np
    import __graft_entry__ as ge
    sps = ge.load_package()
    which = argv[0]
    if which == "svd_left":
        e = sps.Engine(2, 2)
        a = graded(648, 648, 0.03, 5)
        Lm = np.linalg.qr(a.T)[1].T.copy()
        for _ in range(2):
            u, s, sweeps, ms = e.la_svd_left(Lm)
        print(f"svd_left 648x648: {ms:.2f} ms, {sweeps} sweeps")
    elif which == "topk":
        e = sps.Engine(2, 2)
        w = int(argv[1]) if len(argv) > 1 else 1
        gram = len(argv) > 2 and argv[2] == "gram"
        import torch
        sms = torch.cuda.get_device_properties(0).multi_processor_count
        e.set_sm_share(sms // w if w > 1 else 0)
        a = graded(648, 648, 0.1, 5)
        e.la_svd_topk(a, 18, gram=gram, rtol=1e-10 if gram else 0.0)
        e.set_profile(True)
        u, s, v, iters, ms = e.la_svd_topk(a, 18, gram=gram, rtol=1e-10 if gram else 0.0)
        print(f"topk 648x648 k=18 (SM share 1/{w}{', gram' if gram else ''}): {ms:.3f} ms, {iters} iterations")
        for name, st in sorted(e.kernel_stats().items()):
            print(f"  {name:24s} {st['ms']:9.3f} ms  x{st['count']}")
    elif which == "gemm":
        e = sps.Engine(2, 2)
        rng = np.random.default_rng(1)
        a = rng.standard_normal((23328, 648))
        b = rng.standard_normal((648, 648))
        for _ in range(3):
            c, ms = e.la_gemm(a, b)
        print(f"gemm 23328x648x648: {ms:.3f} ms, {2 * 23328 * 648 * 648 / ms / 1e9:.2f} TFLOP/s")
        for _ in range(3):
            g, ms = e.la_gemm(a, a, transpose_a=True)
        print(f"gram 648x648x23328: {ms:.3f} ms, {2 * 23328 * 648 * 648 / ms / 1e9:.2f} TFLOP/s")
    elif which == "tcgemm":
        # the tcgen05 contraction GEMM on dense operands: (m x k) (k x n) in a low-precision mode
        mode = argv[1] if len(argv) > 1 else "3xtf32"
        m, n, k = (int(v) for v in argv[2:5]) if len(argv) > 4 else (8192, 8192, 8192)
        e = sps.Engine(2, 2)
        rng = np.random.default_rng(1)
        a = rng.standard_normal((m, k))
        b = rng.standard_normal((k, n))
        for _ in range(3):
            c, ms = e.la_gemm_mixed(a, b, mode)
        e.set_profile(True)
        c, ms = e.la_gemm_mixed(a, b, mode)
        st = e.kernel_stats()
        e.set_profile(False)
        g = [v for kk, v in st.items() if kk.startswith("tc_gemm")][0]
        passes = 1 if mode == "tf32" else 3
        print(f"tcgemm {mode} {m}x{n}x{k}: pack+gemm {ms:.3f} ms, gemm {g['ms']:.3f} ms, "
              f"{2 * m * n * k / g['ms'] / 1e9:.1f} TFLOP/s effective, {passes * 2 * m * n * k / g['ms'] / 1e9:.1f} "
              f"TFLOP/s on the tensor cores; rel err {np.linalg.norm(c - a @ b) / np.linalg.norm(a @ b):.2e}")
    elif which == "qr":
        e = sps.Engine(2, 2)
        a = np.random.default_rng(3).standard_normal((23328, 648))
        for _ in range(2):
            q, r, ms = e.la_qr(a)
        print(f"qr 23328x648: {ms:.2f} ms")
    elif which in ("draw", "zipdraw"):
        e = sps.Engine(LX, LY, sps.TFIM(1.0, H_FIELD))
        if len(argv) > 1 and argv[1] == "synthetic":   # the seeded synthetic beta0 stand-in of the same shapes
            sites, dims = sps.synthetic.synthetic_pepo(LX, LY, D, PEPO_EPS, PEPO_SEED)
            st = e.upload_state(sites, dims, True, beta=BETA0)
            sps.normalize_state(st)
        else:
            st = purified_state(sps, e)
        kind = sps.BoundaryMPS if which == "draw" else sps.BoundaryMPSZipUp
        cache = sps.SamplingCache(st, kind(CHI, sps.Z2Space(CHI // 2, CHI // 2)))
        for i in range(2):
            if i == 1:
                e.set_profile(2)
                t0 = time.perf_counter()
            d = sps.sample_configuration(cache, uniforms=sps.sample_uniforms(SEED, i + 1, LX * LY))
        wall = (time.perf_counter() - t0) * 1e3
        stats = e.kernel_stats()
        e.set_profile(False)
        dev = sum(v["ms"] for k, v in stats.items() if not k.startswith(("host.", "svd_topk.", "gemm_gather ")))
        print(f"draw log_probability {d['log_probability']}: wall {wall:.1f} ms (profiled), kernels {dev:.1f} ms")
        for name, v in sorted(stats.items(), key=lambda kv: -kv[1]["ms"])[:60]:
            tf = v["flops"] / v["ms"] / 1e9 if v["ms"] > 0 else 0.0
            print(f"  {name:40s} {v['ms']:9.3f} ms  x{v['count']:<5d} {tf:6.2f} TF/s")
    elif which == "scale":
        Ls, Dd, chi = 12, 8, 64
        e = sps.Engine(Ls, Ls, sps.TFIM(1.0, H_FIELD))
        sites, dims = sps.synthetic.synthetic_pepo(Ls, Ls, Dd, PEPO_EPS, 11)
        st = e.upload_state(sites, dims, True, beta=0.5)
        sps.normalize_state(st)
        t = time.perf_counter()
        cache = sps.SamplingCache(st, sps.BoundaryMPSZipUp(chi, sps.Z2Space(chi // 2, chi // 2)))
        print(f"cache {time.perf_counter() - t:.2f} s")
        sps.sample_configuration(cache, uniforms=sps.sample_uniforms(SEED, 1, Ls * Ls))
        t = time.perf_counter()
        d = sps.sample_configuration(cache, uniforms=sps.sample_uniforms(SEED, 2, Ls * Ls))
        print(f"one draw {time.perf_counter() - t:.3f} s, log_probability {d['log_probability']:.6f}")
        w = 4
        e.set_concurrency(w)
        u = np.stack([sps.sample_uniforms(SEED, 10 + j, Ls * Ls) for j in range(2 * w)])
        sps.sample_batch(cache, u[:w])
        t = time.perf_counter()
        sps.sample_batch(cache, u)
        dt = time.perf_counter() - t
        print(f"{2 * w} draws {w} at a time: {dt:.3f} s, {2 * w / dt:.2f} samples/s")
        e.set_concurrency(1)
    elif which == "fustep":
        # one full-update Trotter step of a projected sample and one energy measurement,
        # L x L D=6 chi=36: both absorptions, FP64 and the split-TF32 contractions
        Ls = int(argv[1]) if len(argv) > 1 else LX
        e = sps.Engine(Ls, Ls, sps.TFIM(1.0, H_FIELD))
        if Ls == LX:
            st = purified_state(sps, e)
        else:
            sites, dims = sps.synthetic.synthetic_pepo(Ls, Ls, D, PEPO_EPS, PEPO_SEED)
            st = e.upload_state(sites, dims, True, beta=BETA0)
            sps.normalize_state(st)
        cfg = sps.sample_configuration(sps.SamplingCache(st, sps.BoundaryMPSZipUp(CHI, sps.Z2Space(CHI // 2, CHI // 2))),
                                       uniforms=sps.sample_uniforms(SEED, 1, Ls * Ls))["configuration"]
        for zipup in (True, False):
            for prec in ("fp64", "3xtf32"):
                kind = sps.BoundaryMPSZipUp if zipup else sps.BoundaryMPS
                m = kind(CHI, sps.Z2Space(CHI // 2, CHI // 2))
                ps, _ = sps.project_configuration(st, cfg)
                e.set_precision(prec)
                tag = f"{Ls}x{Ls} {'zip-up' if zipup else 'exact'} {prec}"
                try:
                    e.set_profile(True)
                    t = time.perf_counter()
                    r = sps.evolution_step(ps, DTAU, D, m, sps.Z2Space(D // 2, D // 2))
                    dt = time.perf_counter() - t
                    top = sorted(e.kernel_stats().items(), key=lambda kv: -kv[1]["ms"])[:8]
                    e.set_profile(False)
                    t = time.perf_counter()
                    en = sps.measure_energy(ps, m)
                    dm = time.perf_counter() - t
                    print(f"{tag}: FU step {dt:.2f} s, bond updates {r['bond_updates']}, repairs {r['repairs']}, "
                          f"stops {[r['stop_' + k] for k in ('error_tolerance', 'iteration_limit', 'residual_fallback', 'disabled')]}, "
                          f"measure_energy {dm:.2f} s (E {en['energy_per_site']:.10f}); "
                          + ", ".join(f"{k} {v['ms']:.0f} ms" for k, v in top), flush=True)
                except Exception as ex:
                    e.set_profile(False)
                    print(f"{tag}: {type(ex).__name__}: {ex}", flush=True)
                e.set_precision("fp64")
                del ps
        e.close()
    elif which == "purify":
        # run_purification of the L x L TFIM (h = 3.0) at D=6 chi=36 to beta0 = 0.4 (tau = 0.02), one
        # evolution step at a time within a wall-clock budget; the state reached is saved
        Ls = int(argv[1]) if len(argv) > 1 else LX
        budget = float(argv[2]) if len(argv) > 2 else 600.0
        prec = argv[3] if len(argv) > 3 else "fp64"
        e = sps.Engine(Ls, Ls, sps.TFIM(1.0, H_FIELD))
        e.set_precision(prec)
        st = e.identity_pepo()
        sps.normalize_state(st)
        m = sps.BoundaryMPS(CHI, sps.Z2Space(CHI // 2, CHI // 2))
        t0 = time.perf_counter()
        for beta in sps.step_schedule(0.0, BETA0, DTAU):
            t = time.perf_counter()
            try:
                r = sps.evolution_step(st, (beta - st.beta) / 2, D, m, sps.Z2Space(D // 2, D // 2))
            except Exception as ex:
                print(f"beta {beta}: {type(ex).__name__}: {ex}", flush=True)
                break
            st.beta = beta
            print(f"beta {beta:.2f}: {time.perf_counter() - t:.2f} s, repairs {r['repairs']}, "
                  f"max state truncation {r['max_state_truncation']:.3e}, env truncation "
                  f"{r['max_environment_truncation']:.3e}", flush=True)
            if time.perf_counter() - t0 > budget:
                break
        sites, dims = st.download()
        os.makedirs(os.path.join(ROOT, out), exist_ok=True)
        np.savez_compressed(os.path.join(ROOT, out, f"purified_{Ls}x{Ls}_D{D}_{prec}.npz"),
                            data=np.concatenate([np.asarray(a).reshape(-1) for a in sites]), dims=np.asarray(dims),
                            beta=st.beta, log_amplitude=st.log_amplitude)
        en = sps.measure_energy(st, m)
        print(f"beta {st.beta}: E per site {en['energy_per_site']:.12f}, lnZ {en['log_norm']:.12f}, "
              f"total {time.perf_counter() - t0:.1f} s", flush=True)
    elif which == "adjoint":
        # lognorm, its reverse-mode derivative and the field derivatives on the seeded synthetic PEPO
        Ls = int(argv[1]) if len(argv) > 1 else LX
        Dd = int(argv[2]) if len(argv) > 2 else D
        chi = int(argv[3]) if len(argv) > 3 else CHI
        e = sps.Engine(Ls, Ls, sps.TFIM(1.0, H_FIELD))
        sites, dims = sps.synthetic.synthetic_pepo(Ls, Ls, Dd, PEPO_EPS, PEPO_SEED)
        st = e.upload_state(sites, dims, True, beta=1.0)
        sps.normalize_state(st)
        m = sps.BoundaryMPS(chi, sps.Z2Space(chi // 2, chi // 2))
        # the full tape holds about 4 absorbed-row tensors (chi D^2, D^2, chi D^2) per site for every row
        # (about 130 GB at 8x8 D=6 chi=36); row checkpoints hold one row's
        tape_gb = 4 * 8 * (chi * Dd * Dd) ** 2 * Dd * Dd * Ls * Ls / 1e9
        variants = [("lognorm", lambda: sps.lognorm(st, m)["log_norm"]),
                    ("gradient, row checkpoints", lambda: sps.lognorm_gradient(st, m, checkpoint_rows=True)[0]),
                    ("field gradient, row checkpoints",
                     lambda: sps.lognorm_field_gradient(st, m, checkpoint_rows=True)["log_norm"])]
        if tape_gb < 60:
            variants.append(("gradient, full tape", lambda: sps.lognorm_gradient(st, m)[0]))
        else:
            print(f"full tape skipped: about {tape_gb:.0f} GB", flush=True)
        for label, fn in variants:
            try:
                fn()
                t = time.perf_counter()
                v = fn()
                dt = time.perf_counter() - t
                print(f"{Ls}x{Ls} D={Dd} chi={chi} {label}: {dt:.3f} s, lnZ {v:.12f}", flush=True)
            except Exception as ex:
                print(f"{Ls}x{Ls} D={Dd} chi={chi} {label}: {type(ex).__name__}: {ex}", flush=True)
        e.close()
    else:
        raise SystemExit(f"unknown probe {which}\n{PROBES}")


def main():
    args = parse()
    if args.probe:
        probe(args.probe, args.out)
        return
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    ours_arm(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
