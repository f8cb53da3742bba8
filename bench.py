#!/usr/bin/env python
"""Born samples/s on the 8x8 open TFIM (J=1, h=3.0), D=6 (3+3), chi=36 (18+18).

One step = one perfect Born draw (``sample_configuration``, src/sampling/born.jl:86-163):
eight row absorptions and 64 conditionals from a device-resident SamplingCache
of a seeded synthetic beta0 PEPO with the workload's shapes.  The headline
`value` is the zip-up absorption path (FP64); the plain FP64 path with the
reference's exact LQ + truncated-SVD compression is timed beside it on the same
draw indices (`plain_fp64`, `agreement_vs_plain`).  Every rank draws its own
samples (weak scaling: samples shard with no data-path collective); rank 0
prints one JSON line.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import math
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
METRIC = "Born samples/s at 8x8 D6 χ36: batched mixed-prec vs plain FP64 GPU, ΔE≤1e-4"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=4)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--concurrency", type=int, default=8,
                   help="samples drawn at the same time on one GPU (own stream and workspace each)")
    return p.parse_args()


def workload_config(extra=None):
    c = {"workload": "tfim_8x8_D6_chi36_born_draw", "Lx": LX, "Ly": LY, "J": 1.0, "h": H_FIELD, "D": D,
         "bond_space": [D // 2, D // 2], "chi_sampling": CHI, "sampling_space": [CHI // 2, CHI // 2],
         "pepo": f"synthetic seeded beta0 stand-in (identity + {PEPO_EPS} Gaussian Z2 noise, seed 7)",
         "step": "one Born draw from a device-resident SamplingCache",
         "uniforms": "numpy default_rng([seed, sample_index])", "seed": SEED,
         "l2": "inputs larger than L2 (absorbed boundary tensors ~480 MB each)"}
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


def cpu_row_sample():
    """Time the CPU oracle on one interior row of a Born draw: its absorption
    (absorb + exact LQ sweep + truncated SVD sweep) and its Lx conditionals.
    Returns (seconds per draw extrapolated as Ly rows, seconds measured)."""
    import numpy as np
    from oracle import boundary as bm, model as omd, sampling as osp
    from oracle.z2 import T, leg
    import __graft_entry__ as ge
    syn = ge.load_package().synthetic
    sites, dims = syn.synthetic_pepo(LX, LY, D, PEPO_EPS, 7)
    grid = [[None] * LY for _ in range(LX)]
    for i, (a, ld) in enumerate(zip(sites, dims)):
        grid[i % LX][i // LX] = T(a, [leg(int(p), int(q)) for p, q in ld])
    st = omd.State(LX, LY, grid, 0.4, 0.0, "pepo")
    m = bm.BoundaryMPS(CHI, (CHI // 2, CHI // 2))
    layers = bm.row_layers(st)
    env = bm.trivial_boundary(bm.col(layers, 0), "north")
    env = bm.absorb(env, bm.col(layers, 0), m)           # row 0 (untimed setup)
    bottom = env.tensors   # stand-in south boundary with the legs a row-1 conditional contracts
    t0 = time.perf_counter()
    row = bm.col(layers, 1)
    le, ri = bm.row_environments(env.tensors, row, bottom, side="right")
    left = le[0]
    for x in range(LX):
        cand = [bm.double_layer(osp.project(st[x, 1], k)) for k in (0, 1)]
        raw = [bm.row_scalar(left, env.tensors[x], E, bottom[x], ri[x + 1]) for E in cand]
        if x < LX - 1:
            left = bm.safe_scale(bm.left_step(left, env.tensors[x], cand[0], bottom[x]))
    env = bm.absorb(env, row, m)
    dt = time.perf_counter() - t0
    return dt * LY, dt


def reference_arm(args, rank, world):
    if rank != 0:
        return
    import numpy as np
    cores = os.cpu_count()
    times = []
    for s in range(args.warmup + args.steps):
        per_draw, measured = cpu_row_sample()
        if s >= args.warmup:
            times.append(per_draw)
    value = 1.0 / (sum(times) / len(times))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload_config(),
            "cpu_baseline": {"value": value, "unit": "samples/s", "cores": cores, "kind": "port",
                             "sample": "one interior row of a draw (absorption + 8 conditionals) per step, "
                                       "x8 rows; CPU oracle (NumPy/OpenBLAS FP64) restating the Julia "
                                       "reference, which cannot run here (no Julia)"},
            "e2e": {"value": value, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


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
    sites, dims = sps.synthetic.synthetic_pepo(LX, LY, D, PEPO_EPS, 7)
    st = e.upload_state(sites, dims, True, beta=0.4)
    sps.normalize_state(st)
    space = sps.Z2Space(CHI // 2, CHI // 2)

    def index(step):
        return 1 + rank + world * step

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def measure(method, steps, warmup, profile, batch=1):
        """Device-timed and end-to-end Born draws from a cache built with `method`;
        a step is `batch` draws (concurrent when batch > 1)."""
        cache = sps.SamplingCache(st, method)
        e.set_concurrency(batch)

        def draw(i):
            # draw j of step index i uses the uniforms of sample id i * W + j (W: the zip-up batch)
            ids = [i * W + j for j in range(batch)]
            if batch == 1:
                d = sps.sample_configuration(cache, uniforms=sps.sample_uniforms(SEED, ids[0], LX * LY))
                return [dict(d, uid=ids[0])]
            u = np.stack([sps.sample_uniforms(SEED, k, LX * LY) for k in ids])
            cfg, lp = sps.sample_batch(cache, u)
            return [{"configuration": c, "log_probability": l, "uid": k} for c, l, k in zip(cfg, lp, ids)]

        for s in range(warmup):
            draw(index(s))
        barrier()
        n0, _ = e.counters()
        draws = []
        with Clocks(local_rank) as clk:
            e.timer_start()
            for s in range(steps):
                draws.extend(draw(index(warmup + s)))
            ms = e.timer_stop()
        n1, _ = e.counters()
        barrier()
        # end to end through the public API: host uniforms in, configuration out, wall clock
        t0 = time.perf_counter()
        for s in range(steps):
            draw(index(warmup + steps + s))
        barrier()
        wall = time.perf_counter() - t0
        t = torch.tensor([ms, wall], dtype=torch.float64, device=f"cuda:{local_rank}")
        if dist is not None:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        stats = None
        if profile:   # per-kernel profile of one serial draw (separate pass; not part of the timed number)
            e.set_concurrency(1)
            e.set_profile(True)
            u = sps.sample_uniforms(SEED, index(2 * steps + warmup) * W, LX * LY)
            sps.sample_configuration(cache, uniforms=u)
            stats = e.kernel_stats()
            e.set_profile(False)
        e.set_concurrency(1)
        del cache
        return {"ms": float(t[0]), "wall": float(t[1]), "launches": int(n1 - n0), "clocks": clk.summary(),
                "draws": draws, "stats": stats}

    W = max(1, args.concurrency)
    zip_run = measure(sps.BoundaryMPSZipUp(CHI, space), args.steps, args.warmup, True, W)
    plain_steps = max(1, min(args.steps, 2))
    plain_run = measure(sps.BoundaryMPS(CHI, space), plain_steps, min(args.warmup, 3), False)
    value = world * args.steps * W / (zip_run["ms"] * 1e-3)
    e2e = world * args.steps * W / zip_run["wall"]
    plain_value = world * plain_steps / (plain_run["ms"] * 1e-3)
    plain_e2e = world * plain_steps / plain_run["wall"]
    # the two paths on the same draw indices
    import numpy as np
    same, dlp = 0, 0.0
    # precision of the zip-up path: energy per site of the beta0 state with both
    # absorptions (outside the timed regions)
    en_plain = sps.measure_energy(st, sps.BoundaryMPS(CHI, space))
    en_zip = sps.measure_energy(st, sps.BoundaryMPSZipUp(CHI, space))
    # the two paths on the same uniforms (same sample ids)
    zmap = {d["uid"]: d for d in zip_run["draws"]}
    same, dlp, ncmp = 0, 0.0, 0
    for dp in plain_run["draws"]:
        dz = zmap.get(dp["uid"])
        if dz is None:
            continue
        ncmp += 1
        same += int(np.array_equal(dz["configuration"], dp["configuration"]))
        dlp = max(dlp, abs(dz["log_probability"] - dp["log_probability"]))
    result = None
    if rank == 0:
        stats = zip_run["stats"]
        peak = measure_fp64_peak(torch, f"cuda:{local_rank}")
        tot = sum(v["ms"] for k, v in stats.items() if "." not in k)
        dom = max(((k, v) for k, v in stats.items() if v["flops"] > 0 and "." not in k), key=lambda kv: kv[1]["ms"])
        name, v = dom
        per_launch_flops = v["flops"] / v["count"]
        avg_ms = v["ms"] / v["count"]
        achieved = per_launch_flops / (avg_ms * 1e-3) / 1e12
        traffic = None
        if name == "svd_topk":
            # DRAM bytes per svd_topk launch: an ncu capture of `kernel_probe.py topk 1 gram` (one 648x648
            # block, k = 18, Gram mode as in the zip-up splits) moved 10.57 MB (dram__bytes.sum.per_second
            # 11.35 GB/s x gpu__time_duration.sum 931 us): M, M^T and M M^T (10.1 MB) read about once; a
            # bench launch holds both parity blocks of that size
            traffic = 2 * 10.57e6
        roofline = {"bound": "tensor", "kernel": name, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved / peak, "traffic": traffic,
                    "note": "svd_topk is a latency-bound cooperative kernel (chains of small dependent "
                            "phases, one CTA per SM); FLOPs counted: 2 m n b per product",
                    "peak_source": "FP64: cuBLAS DGEMM 8192^3 measured in this run (FP64 is not in "
                                   "MEASURED_PEAKS.json); tensor-core FP64 and DFMA share the FP64 rate on B200",
                    "share_of_profiled_time": v["ms"] / tot if tot else None,
                    "kernels": {k: {"ms": round(s["ms"], 3), "count": s["count"],
                                    "share": round(s["ms"] / tot, 4) if tot and "." not in k else None,
                                    "tflops": round(s["flops"] / (s["ms"] * 1e-3) / 1e12, 3)
                                    if s["ms"] > 0 and s["flops"] > 0 else None}
                                for k, s in sorted(stats.items(), key=lambda kv: -kv[1]["ms"])}}
        cpu = None
        if world == 1:
            per_draw, measured = cpu_row_sample()
            cpu = {"value": 1.0 / per_draw, "unit": "samples/s", "cores": os.cpu_count(), "kind": "port",
                   "sample": f"one interior row of a draw (absorption + {LX} conditionals) timed "
                             f"({measured:.1f} s) and scaled x{LY}; CPU oracle (NumPy/OpenBLAS FP64), "
                             "reference algorithm"}
        L = LX * LY
        result = {"metric": METRIC, "value": value, "unit": "samples/s", "n_gpus": world, "steps": args.steps,
                  "warmup": args.warmup, "ms_per_step": zip_run["ms"] / args.steps, "higher_is_better": True,
                  "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                  "config": workload_config({"parallelism": f"samples sharded over {world} GPU(s)",
                                             "path": f"zip-up boundary absorption, FP64, {W} samples "
                                                     "concurrently (own stream and workspace each)",
                                             "samples_per_step": W}),
                  "e2e": {"value": e2e, "unit": "samples/s", "h2d_bytes_per_step": 8 * L * W,
                          "d2h_bytes_per_step": (4 * L + 8) * W},
                  "gpu_launches": zip_run["launches"], "clocks": zip_run["clocks"], "roofline": roofline,
                  "cpu_baseline": cpu,
                  "plain_fp64": {"value": plain_value, "e2e": plain_e2e, "unit": "samples/s",
                                 "steps": plain_steps, "ms_per_step": plain_run["ms"] / plain_steps,
                                 "gpu_launches": plain_run["launches"], "clocks": plain_run["clocks"],
                                 "path": "reference algorithm: exact LQ sweep + truncated SVD sweep, FP64"},
                  "speedup_vs_plain_fp64": value / plain_value,
                  "agreement_vs_plain": {"draws": ncmp, "identical_configurations": same,
                                         "max_abs_dlogp": dlp},
                  "precision": {"energy_per_site_plain_fp64": en_plain["energy_per_site"],
                                "energy_per_site_zipup": en_zip["energy_per_site"],
                                "abs_delta_e": abs(en_zip["energy_per_site"] - en_plain["energy_per_site"]),
                                "tolerance": 1e-4,
                                "state": "the synthetic beta0 PEPO of the workload, chi=36 (18+18)"}}
        print(json.dumps(result), flush=True)
    del st
    e.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    ours_arm(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
