"""Run one hot operation of the engine on a representative input, for profiling.

  python stopeps.jl_b200/kernel_probe.py svd_left   # U-only Jacobi of a 648x648 LQ-preconditioned block
  python stopeps.jl_b200/kernel_probe.py qr          # blocked Householder QR of a 23328x648 block
  python stopeps.jl_b200/kernel_probe.py topk [W] [gram]  # leading 18 triplets of a 648x648 graded block (1/W of the SMs)
  python stopeps.jl_b200/kernel_probe.py gemm        # FP64 GEMM 23328x648x648 and the 648x648x23328 Gram
  python stopeps.jl_b200/kernel_probe.py draw        # one Born draw, 8x8 D=6 chi=36 (synthetic PEPO)
  python stopeps.jl_b200/kernel_probe.py zipdraw     # the same draw with the zip-up absorption
  python stopeps.jl_b200/kernel_probe.py scale       # zip-up draws at 12x12 D=8 chi=64 (32+32): 1 and 4 at a time
  python stopeps.jl_b200/kernel_probe.py fustep [L]  # one full-update Trotter step, L x L D=6 chi=36 (default 8)

Each operation runs once to warm up and once more; the sizes are those of the
8x8, D=6, chi=36 boundary compression (parity blocks of 648 and 23328 rows).
Inputs are seeded synthetic matrices with a graded spectrum like the
boundary-MPS Schmidt spectra.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def graded(m, n, decay, seed):
    rng = np.random.default_rng(seed)
    u, _ = np.linalg.qr(rng.standard_normal((m, min(m, n))))
    v, _ = np.linalg.qr(rng.standard_normal((n, min(m, n))))
    return (u * np.exp(-decay * np.arange(min(m, n)))) @ v.T


def main(which):
    import __graft_entry__ as ge
    sps = ge.load_package()
    if which == "svd_left":
        e = sps.Engine(2, 2)
        a = graded(648, 648, 0.03, 5)
        L = np.linalg.qr(a.T)[1].T.copy()
        for _ in range(2):
            u, s, sweeps, ms = e.la_svd_left(L)
        print(f"svd_left 648x648: {ms:.2f} ms, {sweeps} sweeps")
    elif which == "topk":
        e = sps.Engine(2, 2)
        w = int(sys.argv[2]) if len(sys.argv) > 2 else 1
        gram = len(sys.argv) > 3 and sys.argv[3] == "gram"
        import torch
        sms = torch.cuda.get_device_properties(0).multi_processor_count
        e.set_sm_share(sms // w if w > 1 else 0)   # the launch's share of the SMs: 1/w
        a = graded(648, 648, 0.1, 5)
        u, s, v, iters, ms = e.la_svd_topk(a, 18, gram=gram, rtol=1e-10 if gram else 0.0)
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
    elif which == "qr":
        e = sps.Engine(2, 2)
        a = np.random.default_rng(3).standard_normal((23328, 648))
        for _ in range(2):
            q, r, ms = e.la_qr(a)
        print(f"qr 23328x648: {ms:.2f} ms")
    elif which in ("draw", "zipdraw"):
        e = sps.Engine(8, 8, sps.TFIM(1.0, 3.0))
        sites, dims = sps.synthetic.synthetic_pepo(8, 8, 6, 0.15, 7)
        st = e.upload_state(sites, dims, True, beta=0.4)
        sps.normalize_state(st)
        kind = sps.BoundaryMPS if which == "draw" else sps.BoundaryMPSZipUp
        cache = sps.SamplingCache(st, kind(36, sps.Z2Space(18, 18)))
        import time
        for i in range(2):
            if i == 1:
                e.set_profile(2)
                t0 = time.perf_counter()
            d = sps.sample_configuration(cache, uniforms=sps.sample_uniforms(1, i + 1, 64))
        wall = (time.perf_counter() - t0) * 1e3
        stats = e.kernel_stats()
        e.set_profile(False)
        dev = sum(v["ms"] for k, v in stats.items() if not k.startswith(("host.", "svd_topk.", "gemm_gather ")))
        print(f"draw log_probability {d['log_probability']}: wall {wall:.1f} ms (profiled), kernels {dev:.1f} ms")
        for name, v in sorted(stats.items(), key=lambda kv: -kv[1]["ms"])[:60]:
            tf = v["flops"] / v["ms"] / 1e9 if v["ms"] > 0 else 0.0
            print(f"  {name:40s} {v['ms']:9.3f} ms  x{v['count']:<5d} {tf:6.2f} TF/s")
    elif which == "scale":
        import time
        L, Dd, chi = 12, 8, 64
        e = sps.Engine(L, L, sps.TFIM(1.0, 3.0))
        sites, dims = sps.synthetic.synthetic_pepo(L, L, Dd, 0.15, 11)
        st = e.upload_state(sites, dims, True, beta=0.5)
        sps.normalize_state(st)
        t = time.perf_counter()
        cache = sps.SamplingCache(st, sps.BoundaryMPSZipUp(chi, sps.Z2Space(chi // 2, chi // 2)))
        print(f"cache {time.perf_counter() - t:.2f} s")
        d = sps.sample_configuration(cache, uniforms=sps.sample_uniforms(1, 1, L * L))
        t = time.perf_counter()
        d = sps.sample_configuration(cache, uniforms=sps.sample_uniforms(1, 2, L * L))
        print(f"one draw {time.perf_counter() - t:.3f} s, log_probability {d['log_probability']:.6f}")
        for w in (4,):
            e.set_concurrency(w)
            u = np.stack([sps.sample_uniforms(1, 10 + j, L * L) for j in range(2 * w)])
            sps.sample_batch(cache, u[:w])
            t = time.perf_counter()
            sps.sample_batch(cache, u)
            dt = time.perf_counter() - t
            print(f"{2 * w} draws {w} at a time: {dt:.3f} s, {2 * w / dt:.2f} samples/s")
        e.set_concurrency(1)
    elif which == "fustep":
        import time
        L = int(sys.argv[2]) if len(sys.argv) > 2 else 8
        for zipup in (True, False):
            e = sps.Engine(L, L, sps.TFIM(1.0, 3.0))
            sites, dims = sps.synthetic.synthetic_pepo(L, L, 6, 0.15, 7)
            st = e.upload_state(sites, dims, True, beta=0.4)
            sps.normalize_state(st)
            kind = sps.BoundaryMPSZipUp if zipup else sps.BoundaryMPS
            e.set_profile(True)
            t = time.perf_counter()
            r = sps.evolution_step(st, 0.02, 6, kind(36, sps.Z2Space(18, 18)), sps.Z2Space(3, 3))
            dt = time.perf_counter() - t
            top = sorted(e.kernel_stats().items(), key=lambda kv: -kv[1]["ms"])[:6]
            print(f"{L}x{L} {'zip-up' if zipup else 'exact'} environments: {dt:.2f} s, bond updates "
                  f"{r['bond_updates']}, " + ", ".join(f"{k} {v['ms']:.0f} ms" for k, v in top))
            e.close()
    else:
        raise SystemExit(f"unknown operation {which}")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "svd_left")
