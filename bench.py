"""Walker-steps/s of the miniAFQMC walker hot path on B200.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--config C4] [--precision fp64|mixed]

A step is one substep of the driver loop (miniafqmc_base.cpp:251-337: mixed density
matrix, vbias, sigma, vHS, propagation, overlaps, weights; orthogonalisation every
`northo` substeps) plus, every `energy_every` substeps, the mixed density matrix and
local energy (miniafqmc_base.cpp:341-345).  The default workload is the target system:
NMO=384, 48+48 electrons, nchol=1536 Cholesky vectors (20% nonzero), 1024 walkers per
GPU, synthetic (seeded) inputs.  Multi-GPU runs shard walkers (weak scaling): each
rank holds its own 1024 walkers and the per-step Eshift sum is all-reduced.

Rank 0 prints one JSON line.  `value` is whole-job walker-steps/s with the walker set
resident in HBM; `e2e` is the same rate through the C ABI with host buffers (the normals
of every step copied host->device, W_data copied back every step).  `--impl reference`
times the FP64 CPU restatement of the reference (the oracle, with the reference's call
granularity and Release flags) on the host cores, on a bounded sample of walkers.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "walker-steps/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--config", default="C4")
    p.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    p.add_argument("--energy-every", type=int, default=10)
    p.add_argument("--northo", type=int, default=5)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--cpu-walkers", type=int, default=0)
    return p.parse_args()


def workload(cfg, args, nw):
    return {
        "workload": (f"{args.config}: NMO={cfg.nmo}, {cfg.nel}+{cfg.nel} electrons, "
                     f"nchol={cfg.nchol} ({cfg.density:.0%} nonzero), {nw} walkers/GPU, "
                     f"dt={cfg.dt}, Taylor order {cfg.taylor_order}, ortho every {args.northo}, "
                     f"energy every {args.energy_every} substeps (Cholesky form)"),
        "precision": args.precision,
        "l2": "inputs larger than L2 (vHS, walkers, Spvn, SpvnT each > 126 MB); no flush",
        "seed": cfg.seed,
    }


# --------------------------------------------------------------------------- helpers
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 7:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[0]) for r in self.rows if num(r[0]) is not None]
        mx = [num(r[1]) for r in self.rows if num(r[1]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if "Active" in r[3 + i]
                          and "Not" not in r[3 + i]})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        return json.load(open(path)), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def fp64_peak_tflops(torch):
    """The FP64 roofline denominator: cuBLAS DGEMM 8192^3 via torch.matmul, best of 5
    (no FP64 figure is provided in MEASURED_PEAKS.json)."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    b = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    best = 1e9
    for _ in range(6):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    return 2 * 8192 ** 3 / (best * 1e-3) / 1e12


def stage_flops(cfg, nw, stage, order=6):
    """Algorithmic FLOPs (complex multiply-add = 8 FLOP) of one call of a stage."""
    N, n, nc = cfg.nmo, cfg.nel, cfg.nchol
    d = cfg.density
    if stage == "propagate":     # (order + 2) GEMMs of N x N x 2n per walker
        return 8.0 * nw * (order + 2) * N * N * 2 * n
    if stage == "vbias":         # dense SpvnT: nchol x 2nN per walker
        return 8.0 * nw * nc * 2 * n * N
    if stage == "vHS":           # real Spvn (nnz) x complex X
        return 4.0 * nw * d * N * N * nc
    if stage == "DM":
        return 8.0 * nw * 2 * (2 * n * n * N + n ** 3)
    if stage == "energy":        # Coulomb + exchange per walker
        return 8.0 * nw * (2 * n * N * nc + 2 * nc * n * n * N)
    return 0.0


# --------------------------------------------------------------------------- CPU leg
def cpu_rate(system, cfg, args, nwalk_sample, threads):
    """walker-steps/s of the oracle (reference-structured FP64 CPU path, Release flags)
    on `nwalk_sample` walkers: 2 substeps + one energy evaluation, amortised like the
    GPU run (one energy every energy_every substeps)."""
    from oracle import oracle as O
    try:
        from threadpoolctl import threadpool_limits
        lim = threadpool_limits(limits=1)
    except Exception:
        lim = None
    o = O.Oracle(system, nwalk_sample, fast=True, threads=threads)
    o.calculate_mixed_density_matrix()
    t0 = time.perf_counter()
    ksub = 2
    for st in range(ksub):
        o.substep(cfg.seed, st, args.northo)
    t1 = time.perf_counter()
    o.calculate_mixed_density_matrix()
    o.calculate_energy("chol")
    t2 = time.perf_counter()
    if lim is not None:
        lim.unregister() if hasattr(lim, "unregister") else None
    per_step = (t1 - t0) / ksub + (t2 - t1) / args.energy_every
    return nwalk_sample / per_step, {
        "substep_s": (t1 - t0) / ksub, "energy_s": t2 - t1,
        "sample": f"{nwalk_sample} walkers of the same system, {ksub} substeps + 1 energy "
                  f"(amortised over {args.energy_every} substeps), OpenMP over walkers"}


def run_reference(args):
    from miniafqmc_b200.synthetic import CONFIGS, make_system
    import dataclasses
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg = dataclasses.replace(CONFIGS[args.config], with_vakbl=False)
    s = make_system(cfg)
    threads = os.cpu_count() or 1
    nws = args.cpu_walkers or max(threads, 8)
    rates = []
    for _ in range(max(1, min(args.steps, 2))):
        r, info = cpu_rate(s, cfg, args, nws, threads)
        rates.append(r)
    v = float(np.median(rates))
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": METRIC,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic", "config": workload(cfg, args, cfg.nwalk),
        "cpu_baseline": {"value": v, "unit": METRIC, "cores": threads, "kind": "port",
                         "sample": info["sample"]},
        "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- GPU leg
def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    from miniafqmc_b200.afqmc import AfqmcSys, AFQ_PREC_FP64, AFQ_PREC_MIXED
    from miniafqmc_b200.synthetic import CONFIGS, make_system
    from miniafqmc_b200 import driver
    import dataclasses
    cfg = dataclasses.replace(CONFIGS[args.config], with_vakbl=False)
    s = make_system(cfg)
    nw = cfg.nwalk
    prec = AFQ_PREC_MIXED if args.precision == "mixed" else AFQ_PREC_FP64
    eng = AfqmcSys(s, nw, precision=prec, device=local, use_vakbl=False)
    comm = None
    if world > 1:
        def allreduce(vals):
            t = torch.tensor(vals, dtype=torch.float64, device="cuda")
            dist.all_reduce(t)
            return t.tolist()
        comm = driver.Comm(rank * nw, world * nw, allreduce)
        eng.set_walker_offset(rank * nw, world * nw)
    stream = torch.cuda.ExternalStream(eng.stream)

    def one_step(st):
        driver.substep(eng, cfg.seed, st, args.northo, comm, graph=False)
        if (st + 1) % args.energy_every == 0:
            eng.calculate_mixed_density_matrix()
            driver.energy(eng, "chol", comm)

    eng.calculate_mixed_density_matrix()
    driver.energy(eng, "chol", comm)
    for st in range(args.warmup):
        one_step(st)
    eng.synchronize()
    eng.stage_times(reset=True)
    eng.profile(True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for st in range(args.warmup, args.warmup + args.steps):
            one_step(st)
        e1.record(stream)
        eng.synchronize()
        torch.cuda.synchronize()
    eng.profile(False)
    ms = e0.elapsed_time(e1)
    stages = eng.stage_times(reset=True)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    value = world * nw * args.steps / (ms * 1e-3)
    launches = int(sum(v[1] for v in stages.values()))

    # ---- end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        K = args.steps
        xs = torch.empty((K, cfg.nchol, nw), dtype=torch.float64, pin_memory=True)
        g = torch.Generator().manual_seed(cfg.seed)
        xs.normal_(generator=g)
        wd = torch.empty((nw, 8, 2), dtype=torch.float64, pin_memory=True)
        xnp, wdnp = xs.numpy(), wd.numpy()
        import ctypes
        eng.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k in range(K):
            st = args.warmup + args.steps + k
            eng.calculate_mixed_density_matrix()
            eng.get_vbias()
            eng._check(eng.lib.afq_sigma_from(eng.h, ctypes.c_void_p(xnp[k].ctypes.data)))
            eng.get_vHS()
            eng.propagate()
            eng.calculate_overlaps(save_old=True)
            if comm is None:
                eng.update_weights()
            else:
                tot = comm.allreduce([eng.update_weights_partial()])[0]
                eng.eshift = tot / comm.nwalk_global
            if st > 0 and st % args.northo == 0:
                eng.orthogonalize()
                eng.calculate_overlaps()
            if (k + 1) % args.energy_every == 0:
                eng.calculate_mixed_density_matrix()
                driver.energy(eng, "chol", comm)
            eng._check(eng.lib.afq_get_walkers(eng.h, None, ctypes.c_void_p(wdnp.ctypes.data)))
        eng.synchronize()
        t_e2e = time.perf_counter() - t0
        if world > 1:
            t = torch.tensor([t_e2e], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            t_e2e = float(t.item())
        e2e = {"value": world * nw * K / t_e2e, "unit": METRIC,
               "h2d_bytes_per_step": int(cfg.nchol * nw * 8),
               "d2h_bytes_per_step": int(nw * 8 * 16),
               "note": "per step: normals H2D (pinned) via afq_sigma_from, W_data D2H via afq_get_walkers"}

    if rank != 0:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    # ---- roofline of the dominant stage
    peaks, src = measured_peaks()
    dom = max(stages, key=lambda k: stages[k][0])
    dom_ms, dom_launch = stages[dom]
    calls = {"propagate": args.steps, "vbias": args.steps, "vHS": args.steps,
             "DM": args.steps + args.steps // args.energy_every,
             "energy": args.steps // args.energy_every}.get(dom, args.steps)
    flops = stage_flops(cfg, nw, dom) * calls
    if args.precision == "fp64":
        peak = fp64_peak_tflops(torch)
        peak_src = "FP64 cuBLAS DGEMM 8192^3 measured in this run (no FP64 entry in MEASURED_PEAKS.json)"
    else:
        peak = peaks["bf16_tflops_sustained"]
        peak_src = f"bf16 sustained, {src}"
    achieved = flops / (dom_ms * 1e-3) / 1e12 if dom_ms > 0 else 0.0
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get(f"{args.config}:{args.precision}:{dom}")
    roof = {"kernel": dom, "bound": "tensor" if args.precision == "mixed" else "fp64",
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "traffic": traffic, "peak_source": peak_src,
            "avg_launch_ms": dom_ms / max(dom_launch, 1), "launches": dom_launch}

    cpu = None
    if not args.no_cpu and world == 1:
        threads = os.cpu_count() or 1
        r, info = cpu_rate(s, cfg, args, args.cpu_walkers or max(threads, 8), threads)
        cpu = {"value": r, "unit": METRIC, "cores": threads, "kind": "port",
               "sample": info["sample"]}

    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "bf16/tf32+f64",
        "data": "synthetic", "config": workload(cfg, args, nw),
        "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
        "clocks": clk.summary(),
        "stages_ms": {k: round(v[0], 3) for k, v in stages.items()},
    }
    print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
