"""Walker-steps/s of the miniAFQMC walker hot path on B200.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--config C4] [--form mixed-cv|mixed|fp64] [--no-fp64]

A step is one substep of the driver loop (miniafqmc_base.cpp:251-337: mixed density
matrix, vbias, sigma, vHS, propagation, overlaps, weights; orthogonalisation every
`northo` substeps) plus, every `energy_every` substeps, the mixed density matrix and the
local energy (miniafqmc_base.cpp:341-345).  The workload is the target system: NMO=384,
48+48 electrons, nchol=1536 Cholesky vectors (20% nonzero), 1024 walkers per GPU,
synthetic seeded inputs.  Multi-GPU runs shard walkers (weak scaling): each rank holds
its own 1024 walkers; the per-substep Eshift sum is all-reduced on the device (NCCL on the
handle's stream between the two graph launches of afq_substep_begin / afq_substep_end) and
the two energy sums on the host at each measurement.

The headline form is mixed precision with the learned control variate (tensor-core
contractions, FP64 LU/QR/weights, exact exchange on 1/8 of the walkers); at N=1 the plain
FP64 form runs the same steps on the same auxiliary fields for the comparison the metric
asks for: speed-up, |dE| between the two forms' mean energies, and energy error per
wall-second sigma_E * sqrt(T) of each (sigma_E from the walker-population variance of
the weighted mean at each measurement, combined over measurements).

Rank 0 prints one JSON line.  `value` is whole-job walker-steps/s with the walker set
resident in HBM, timed over K substeps launched as CUDA graphs (`afq_substep`) with the
energy measurements op by op; `stages_ms` comes from a second pass of K further substeps
op by op with per-stage CUDA events; `e2e` is the same rate through the C ABI with host
buffers (the normals of every step copied host->device, W_data copied back every step).
The control variate's warm-up (its first 2000 exact samples) runs before the timed
region; the same-walker comparison measures the mixed form's final walkers with both
forms.  `--impl reference`
times the FP64 CPU restatement of the reference (the oracle: the reference's call
granularity and GNU Release flags) on the host cores, on a bounded sample of walkers.
"""
from __future__ import annotations

import argparse
import ctypes
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
    p.add_argument("--steps", type=int, default=40)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--config", default="C4")
    p.add_argument("--form", default="mixed-cv", choices=["mixed-cv", "mixed", "fp64"])
    p.add_argument("--energy-every", type=int, default=5)
    p.add_argument("--northo", type=int, default=5)
    p.add_argument("--branch", type=int, default=0,
                   help="1: population control (comb) after every energy measurement (default "
                        "0: none, as in the reference miniapp)")
    p.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison run")
    p.add_argument("--cv-base", type=int, default=0,
                   help="headline control variate: 0 = network on the step's features, 1 = "
                        "plain-bf16 exchange of every walker as the surrogate's base with a "
                        "learned residual (the accuracy pass measures both)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--cpu-walkers", type=int, default=0)
    p.add_argument("--walkers", type=int, default=0, help="walkers per GPU (default: config)")
    p.add_argument("--acc-substeps", type=int, default=500,
                   help="substeps of the energy-accuracy pass (0 skips it)")
    p.add_argument("--acc-equil", type=int, default=100,
                   help="equilibration substeps left out of the accuracy statistics")
    return p.parse_args()


def workload(cfg, args, nw):
    return {
        "workload": (f"{args.config}: NMO={cfg.nmo}, {cfg.nel}+{cfg.nel} electrons, "
                     f"nchol={cfg.nchol} ({cfg.density:.0%} nonzero), {nw} walkers/GPU, "
                     f"dt={cfg.dt}, Taylor order {cfg.taylor_order}, ortho every {args.northo}, "
                     f"energy every {args.energy_every} substeps"),
        "form": args.form,
        "control_variate": (None if args.form != "mixed-cv" else
                            "two-level: plain-bf16 exchange of every walker + learned residual"
                            if args.cv_base else
                            "network on the step's features, exact exchange on 1/8 of the "
                            "walkers"),
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
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if "Active" in r[3 + i] and "Not" not in r[3 + i]})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        return json.load(open(path)), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def fp64_peak_tflops(torch):
    """FP64 roofline denominator: cuBLAS DGEMM 8192^3 via torch.matmul, best of 6
    (MEASURED_PEAKS.json has no FP64 entry)."""
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


def fp64_stage_flops(cfg, nw, stage, order=6):
    """Algorithmic FLOPs of one call of an FP64 stage (complex multiply-add = 8 FLOP)."""
    N, n, nc = cfg.nmo, cfg.nel, cfg.nchol
    if stage == "propagate":
        return 8.0 * nw * (order + 2) * N * N * 2 * n
    if stage == "vbias":
        return 8.0 * nw * nc * 2 * n * N
    if stage == "vHS":
        return 4.0 * nw * cfg.density * N * N * nc
    if stage == "DM":
        return 8.0 * nw * 2 * (2 * n * n * N + n ** 3)
    if stage == "energy":
        return 8.0 * nw * (2 * n * N * nc + 2 * nc * n * n * N)
    return 0.0


def mixed_propagate_bytes(cfg, nw, order=6, preal=True):
    """HBM bytes one mixed-form propagation stage must move with its operand layouts:
    the FP64 walkers in and out, and per product the bf16 operands read once (hi, plus lo
    for the split products), the fp32 Taylor sum read and written, and the next bf16
    operand written (hi, plus lo when the next product is split).  With a real Propg1
    (preal) the P W and P S products read B operands of K = N (separate Re / Im rows)
    instead of 2N.  The last product W = P S also writes the new walkers' T1 operand (rows
    (re, -im), hi + lo) and their next P W operand, so the chain has no pack of W."""
    N, n = cfg.nmo, cfg.nel
    W64 = nw * N * 2 * n * 16            # FP64 walkers
    F = nw * 4 * n * 2 * N * 2           # one bf16 part of a B operand
    Fp = F // 2 if preal else F          # B operand of P W / P S
    V = nw * N * 2 * N * 2               # one bf16 part of the V operand
    S = nw * N * 2 * n * 8               # fp32 Taylor sum
    split = {"P": True, "V1": True, "Vk": False}
    tot = 2 * Fp + S + 2 * F             # S = P W (split): B hi+lo in, S out, next B out
    for k in range(1, order + 1):
        sp = split["V1"] if k == 1 else split["Vk"]
        nxt = 2 * Fp if k == order else (2 * F if split["Vk"] else F)
        tot += V * (2 if sp else 1) + F * (2 if sp else 1) + 2 * S + nxt
    tot += 2 * Fp + W64 + F + 2 * Fp     # W = P S (split), T1 operand, next P W operand
    return float(tot)


def prop_flops(cfg, nw, order=6):
    """Algorithmic FLOPs of one propagation (a6): per walker (order + 2) N x N times N x 2n
    complex products = 16 N^2 n complex multiply-adds at order 6, 8 FLOP each."""
    return 8.0 * nw * (order + 2) * cfg.nmo * cfg.nmo * 2 * cfg.nel


def prop_compulsory_bytes(cfg, nw, preal=True):
    """HBM bytes a propagation cannot avoid in the mixed form's layouts: V (bf16 hi + lo,
    read once for all Taylor terms), the packed P W operand in (hi + lo), the FP64 walkers
    out and the two packed forms of the new walkers out (T1 operand and next P W operand,
    hi + lo)."""
    N, n = cfg.nmo, cfg.nel
    V = 2 * N * 2 * N * 2                 # hi + lo of [N][2N] bf16
    Fp = 4 * n * (N if preal else 2 * N) * 2   # one part of a P-product B operand
    T1op = 2 * n * 2 * N * 2 * 2          # hi + lo of the T1 operand, rows (re, -im)
    W64 = N * 2 * n * 16
    return float(nw * (V + 2 * Fp + W64 + T1op + 2 * Fp))


def mixed_stage_flops(cfg, nw, stage, real_ops=True, subset=None):
    """Algorithmic FLOPs of one call of a mixed-form tensor-core stage (complex x complex
    multiply-add = 8 FLOP, real x complex = 4).  vHS counts the N(N+1)/2 symmetric pairs
    the dense product evaluates; the energy stage counts the exchange of `subset` walkers
    and the Coulomb vectors of all walkers.  Split precision executes three tensor-core
    products per algorithmic product."""
    N, n, nc = cfg.nmo, cfg.nel, cfg.nchol
    nak = 2 * n * N
    f = 4.0 if real_ops else 8.0
    if stage == "vHS":
        return 4.0 * nw * (N * (N + 1) // 2) * nc
    if stage == "vbias":
        return f * nw * nc * nak
    if stage == "energy":
        m = subset if subset is not None else nw
        return f * nw * nc * nak + f * m * 2 * nc * n * n * N
    if stage in ("DM", "overlap"):
        return 8.0 * nw * 2 * (n * n * N + (n * n * N if stage == "DM" else 0))
    return fp64_stage_flops(cfg, nw, stage)


# --------------------------------------------------------------------------- CPU leg
def cpu_rate(system, cfg, args, nwalk_sample, threads):
    """walker-steps/s of the oracle (reference-structured FP64 CPU path, Release flags)
    on `nwalk_sample` walkers: 2 substeps + one exact energy evaluation amortised over
    energy_every substeps, OpenMP over walkers."""
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
    del lim
    per_step = (t1 - t0) / ksub + (t2 - t1) / args.energy_every
    return nwalk_sample / per_step, {
        "sample": f"{nwalk_sample} walkers of the same system, {ksub} substeps + 1 exact energy "
                  f"(amortised over {args.energy_every} substeps), OpenMP over walkers"}


def run_reference(args):
    from miniafqmc_b200.synthetic import CONFIGS, make_system
    import dataclasses
    if int(os.environ.get("RANK", "0")) != 0:
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
class Form:
    """One walker set in one numerical form, with its step loop."""

    def __init__(self, system, cfg, args, form, device, comm, torch, cv_base=None):
        from miniafqmc_b200.afqmc import AfqmcSys, AFQ_PREC_FP64, AFQ_PREC_MIXED
        self.cfg, self.args, self.form, self.comm = cfg, args, form, comm
        prec = AFQ_PREC_FP64 if form == "fp64" else AFQ_PREC_MIXED
        self.eng = AfqmcSys(system, cfg.nwalk, precision=prec, device=device, use_vakbl=False)
        if comm is not None:
            self.eng.set_walker_offset(comm.offset, comm.nwalk_global)
        self.mode = "cv" if form == "mixed-cv" else "chol"
        if self.mode == "cv":
            self.eng.cv_configure(hidden=256, lr=1e-3, seed=cfg.seed, train_walker_steps=2000,
                                  subset_den=8)
            self.cv_base = args.cv_base if cv_base is None else cv_base
            if self.cv_base:   # plain-bf16 exchange of every walker + learned residual
                self.eng.cv_set_base(1)
        self.stream = torch.cuda.ExternalStream(self.eng.stream)
        self.energies, self.sig2, self.cvvar = [], [], []

    def measure(self, record=True):
        from miniafqmc_b200 import driver
        e = self.eng
        e.calculate_mixed_density_matrix()
        E = driver.energy(e, self.mode, self.comm)
        if record:
            Wd = e.get_walker_data()
            w = Wd[:, 1].real
            el = Wd[:, 0].real
            self.energies.append(E)
            s2 = float(np.sum(w * w * (el - E) ** 2) / np.sum(w) ** 2)
            if self.mode == "cv":   # plus the sampling variance of the subset correction
                v = e.cv_stats()["subset_var"]
                s2 += v
                self.cvvar.append(v)
            self.sig2.append(s2)
        return E

    def step(self, st, record=True, graph=True):
        from miniafqmc_b200 import driver
        # sharded runs keep graph substeps with the Eshift sum all-reduced on the device
        driver.substep(self.eng, self.cfg.seed, st, self.args.northo, self.comm, graph=graph)
        if (st + 1) % self.args.energy_every == 0:
            self.measure(record)
            if self.args.branch:   # where the miniapp marks branching (miniafqmc_base.cpp:347)
                self.eng.population_control(self.cfg.seed, st + 1)


def blocking_sigma(x):
    """Standard error of the mean of a correlated series by blocking (Flyvbjerg and
    Petersen, J. Chem. Phys. 91, 461 (1989)): neighbouring values are averaged in pairs
    level after level, the naive standard error of each level's blocks is computed, and
    the largest over the levels that keep at least 8 blocks is returned -- the plateau
    value, or a bound above it when the series is too short to reach the plateau.
    Returns (sigma, per-level sigmas)."""
    x = np.asarray(x, dtype=np.float64)
    levels = []
    while len(x) >= 8:
        n = len(x)
        levels.append(float(np.sqrt(np.var(x, ddof=1) / n)))
        h = n // 2 * 2
        x = 0.5 * (x[0:h:2] + x[1:h:2])
    return (max(levels) if levels else float("nan")), levels


def accuracy_pass(system, cfg, args, device, torch):
    """Energy accuracy at the target run length, apart from the headline timing: four
    walker sets start from the trial and take `acc_substeps` substeps (CUDA-graph
    substeps) on the same Philox fields -- mixed precision with the control variate (the
    headline form), the same with the other control-variate setting, mixed precision with
    exact exchange, and FP64 -- measuring the energy
    every energy_every substeps.  The control variate trains on its first exact samples
    inside the pass (its first measurements are exact on every walker).  Measurements of
    the first `acc_equil` substeps (equilibration from the trial) are left out of the
    statistics.  Per form: mean energy, its standard error by blocking and the device time
    of the whole pass (CUDA events on the form's stream around all its substeps and
    measurements).  |dE| of each mixed form against FP64 on the same fields with the
    blocked standard error of the difference series, and the energy error per wall-second
    sigma_E * sqrt(T) of each form.

    The trajectories of different forms drift apart even on the same fields (the walker
    dynamics amplifies any rounding difference), so the precision of the mixed form is
    measured on identical walkers as well: at every measurement of the FP64 trajectory a
    mixed-form handle with its own control variate takes a device copy of the FP64
    walkers (afq_copy_walkers) and measures them with the control-variate estimator and
    with exact exchange ("same_walkers": the mean difference from FP64, the standard error
    of that mean, the largest single difference; the shadow's time is left out of the FP64
    pass's device time).  Both control-variate settings are measured: the headline's
    (--cv-base) and the other one, as a fourth trajectory and a second shadow."""
    out = {"substeps": args.acc_substeps, "energy_every": args.energy_every,
           "equilibration_substeps": args.acc_equil, "forms": {}}
    series = {}
    # control variates measured on the FP64 trajectory's walkers: the headline's, the other
    # base setting's, and exact exchange
    other = "cv_two_level" if not args.cv_base else "cv_features_only"
    shadow_e = {"cv": [], other: [], "exact": []}
    forms = [("mixed-cv", None), ("mixed-cv-other", 1 - args.cv_base), ("mixed", None),
             ("fp64", None)]
    for name, base in forms:
        kind = "mixed-cv" if name.startswith("mixed-cv") else name
        f = Form(system, cfg, args, kind, device, None, torch, cv_base=base)
        shadows = {}
        if name == "fp64":
            shadows = {"cv": Form(system, cfg, args, "mixed-cv", device, None, torch),
                       other: Form(system, cfg, args, "mixed-cv", device, None, torch,
                                   cv_base=1 - args.cv_base)}
        t_shadow = 0.0
        e = f.eng
        e.synchronize()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(f.stream)
        f.measure(record=False)
        steps = []
        for st in range(args.acc_substeps):
            f.step(st)
            if (st + 1) % args.energy_every == 0:
                steps.append(st + 1)
                if shadows:
                    ts = time.perf_counter()
                    for k, sh in shadows.items():
                        se = sh.eng
                        se.copy_walkers_from(e)
                        se.calculate_mixed_density_matrix()
                        shadow_e[k].append(se.calculate_energy("cv"))
                        if k == "cv":
                            shadow_e["exact"].append(se.calculate_energy("chol"))
                        se.synchronize()
                    t_shadow += time.perf_counter() - ts
        e.synchronize()
        e1.record(f.stream)
        torch.cuda.synchronize()
        secs = e0.elapsed_time(e1) * 1e-3 - t_shadow
        for k, sh in shadows.items():
            out["same_walkers_%s_stats" % k] = sh.eng.cv_stats()
            sh.eng.close()
        keep = np.array(steps) > args.acc_equil
        E = np.array(f.energies)[keep]
        sig, lev = blocking_sigma(E)
        key = name if name != "mixed-cv-other" else "mixed-" + other.replace("_", "-")
        series[key] = E
        rec = {"mean_E": float(E.mean()), "sigma_E_blocked": sig,
               "sigma_E_levels": [float(v) for v in lev], "device_s": secs,
               "measurements": int(keep.sum()), "eps_Ha_sqrt_s": sig * float(np.sqrt(secs))}
        if f.mode == "cv":   # sampling variance of the subset correction, per measurement
            sv = np.array(f.cvvar)[keep]
            rec["subset_sigma_per_measurement_Ha"] = float(np.sqrt(np.mean(sv)))
            rec["control_variate"] = e.cv_stats()
            rec["low_precision_base"] = bool(f.cv_base)
        out["forms"][key] = rec
        e.close()
    for name in series:
        if name == "fp64":
            continue
        d = series[name] - series["fp64"]
        sd, _ = blocking_sigma(d)
        out[f"dE_{name}_vs_fp64"] = {"abs_dE_Ha": float(abs(d.mean())), "sigma_Ha": sd,
                                     "max_abs_per_measurement_Ha": float(np.max(np.abs(d)))}
    keep = np.array(steps) > args.acc_equil
    same = {}
    for k in shadow_e:
        d = np.array(shadow_e[k])[keep] - series["fp64"]
        same[k] = {"dE_Ha": float(d.mean()), "abs_dE_Ha": float(abs(d.mean())),
                   "sigma_of_mean_Ha": float(d.std(ddof=1) / np.sqrt(len(d))),
                   "sigma_of_mean_blocked_Ha": blocking_sigma(d)[0],
                   "rms_per_measurement_Ha": float(np.sqrt(np.mean(d ** 2))),
                   "max_abs_per_measurement_Ha": float(np.max(np.abs(d)))}
    out["same_walkers_along_fp64_trajectory"] = same
    fm, f6 = out["forms"]["mixed-cv"], out["forms"]["fp64"]
    # |dE| of the headline form against FP64 on identical auxiliary fields: the difference
    # of the two trajectories' mean energies, with the blocked standard error of the
    # difference series.  Different forms' trajectories decorrelate within tens of
    # substeps (any rounding difference is amplified through the force bias), so they
    # agree only within that statistical error (z-score beside it).  The precision of the
    # estimator itself shows on identical walkers: its estimate minus FP64's on the FP64
    # trajectory's walkers, averaged over the measurements, with the standard error of
    # that mean (the larger of the naive and the blocked estimate).
    tr = out["dE_mixed-cv_vs_fp64"]
    out["abs_dE_Ha"] = tr["abs_dE_Ha"]
    out["abs_dE_sigma_Ha"] = tr["sigma_Ha"]
    out["abs_dE_z"] = tr["abs_dE_Ha"] / tr["sigma_Ha"] if tr["sigma_Ha"] > 0 else None
    out["abs_dE_definition"] = ("difference of the mean energies of the headline form's and "
                                "the FP64 form's trajectories on the same Philox fields after "
                                "equilibration; sigma = blocked standard error of the "
                                "difference series")
    out["same_walkers_abs_dE_Ha"] = same["cv"]["abs_dE_Ha"]
    out["same_walkers_abs_dE_sigma_Ha"] = max(same["cv"]["sigma_of_mean_Ha"],
                                              same["cv"]["sigma_of_mean_blocked_Ha"])
    # the expectation of the control-variate estimate is the mixed form's exact-exchange
    # energy (the subset correction is unbiased): its deterministic error against FP64
    out["abs_dE_deterministic_Ha"] = same["exact"]["abs_dE_Ha"]
    fo = out["forms"]["mixed-" + other.replace("_", "-")]
    out["other_control_variate"] = {
        "form": other, "abs_dE_Ha": same[other]["abs_dE_Ha"],
        "abs_dE_sigma_Ha": max(same[other]["sigma_of_mean_Ha"],
                               same[other]["sigma_of_mean_blocked_Ha"]),
        "device_s": fo["device_s"], "fp64_over_form": f6["eps_Ha_sqrt_s"] / fo["eps_Ha_sqrt_s"]}
    out["err_per_wall_s"] = {
        "form": fm["eps_Ha_sqrt_s"], "fp64": f6["eps_Ha_sqrt_s"],
        "fp64_over_form": f6["eps_Ha_sqrt_s"] / fm["eps_Ha_sqrt_s"],
        "definition": "sigma_E * sqrt(T): sigma_E the blocked standard error of the mean "
                      "energy over the pass after equilibration, T the device seconds of the "
                      "whole pass (substeps and measurements) of that form"}
    return out


def timed(form, steps, start, torch, dist, world, profile=False, record=True):
    """Times `steps` substeps from step index `start`.  profile=False: CUDA-graph substeps
    (the headline); profile=True: op-by-op calls with per-stage events (the breakdown)."""
    e = form.eng
    e.synchronize()
    e.stage_times(reset=True)
    e.profile(profile)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    torch.cuda.nvtx.range_push("timed")   # `ncu --nvtx --nvtx-include timed/` selects it
    e0.record(form.stream)
    for st in range(start, start + steps):
        form.step(st, record=record, graph=not profile)   # stage events need op-by-op calls
    # the control variate's online training runs on its own stream after each measurement;
    # wait for it (afq_synchronize) so the region holds the last one too, then close it
    e.synchronize()
    e1.record(form.stream)
    torch.cuda.nvtx.range_pop()
    e.synchronize()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    e.profile(False)
    ms = e0.elapsed_time(e1)
    stages = e.stage_times(reset=True)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms, wall, stages


def run_c5(args, torch):
    """Heterogeneous batch (three systems of uneven NMO, electron count and nchol, mixed
    form, one control variate each): K substeps advanced as one CUDA-graph launch per
    substep for all systems (AfqmcBatch), against the fused batch (the vHS product and each
    propagation product one launch over all systems' tiles), the same systems each
    launching its own substep graph on its own stream (independent) and one after another
    with a synchronisation between systems (serial).  Energies every energy_every substeps.
    Times are wall clock around device-synchronised loops (several streams)."""
    from miniafqmc_b200.synthetic import C5_SYSTEMS, make_system
    from miniafqmc_b200.afqmc import AfqmcSys, AfqmcBatch, AFQ_PREC_MIXED
    from miniafqmc_b200 import driver
    systems = [(c, make_system(c)) for c in C5_SYSTEMS]
    nws = [c.nwalk for c, _ in systems]
    seeds = [c.seed for c, _ in systems]

    def fresh():
        engs = []
        for c, sy in systems:
            e = AfqmcSys(sy, c.nwalk, precision=AFQ_PREC_MIXED, use_vakbl=False)
            e.cv_configure(hidden=256, lr=1e-3, seed=c.seed, train_walker_steps=2000, subset_den=8)
            e.calculate_mixed_density_matrix()
            driver.energy(e, "cv", None)
            engs.append(e)
        return engs

    def measure(engs):
        return [driver.energy(e, "cv", None) for e in engs]

    def warm(engs, step_fn):
        st = 0
        while st < args.warmup or any(not e.cv_stats()["active"] for e in engs) or \
                st % args.energy_every:
            step_fn(st)
            st += 1
            if st % args.energy_every == 0:
                for e in engs:
                    e.calculate_mixed_density_matrix()
                measure(engs)
        return st

    def run(mode):
        engs = fresh()
        batch = AfqmcBatch(engs) if mode.startswith(("batch", "fused")) else None
        if mode.startswith("fused"):
            batch.set_fused({"fused": 3, "fused_vhs": 1, "fused_chain": 2}[mode])

        def step(st):
            if batch is not None:   # one launch per measurement interval
                if st % args.energy_every == 0:
                    batch.substeps(seeds, st, args.energy_every, args.northo)
                return
            for e, sd in zip(engs, seeds):
                e.substep(sd, st, args.northo, graph=True)
                if mode == "serial":
                    e.synchronize()

        st0 = warm(engs, step)
        if batch is not None:
            batch.synchronize()
        for e in engs:
            e.synchronize()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for st in range(st0, st0 + args.steps):
            step(st)
            if (st + 1) % args.energy_every == 0:
                for e in engs:
                    e.calculate_mixed_density_matrix()
                measure(engs)
        if batch is not None:
            batch.synchronize()
        for e in engs:
            e.synchronize()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        cv = [e.cv_stats() for e in engs]
        tun = [e.tuning() for e in engs]
        if batch is not None:
            batch.close()
        for e in engs:
            e.close()
        return sum(nws) * args.steps / wall, wall, cv, tun

    res = {m: run(m) for m in ("batch", "fused", "fused_vhs", "fused_chain", "independent",
                               "serial")}
    v, wall, cv, tun = res["batch"]
    line = {
        "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": wall * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16 split/plain tensor-core + f64 LU/QR/weights", "data": "synthetic",
        "config": {"workload": "C5: three systems batched, (NMO 96, 12+12 e, nchol 384, "
                               "128 walkers), (200, 40+40, 800, 256), (320, 64+64, 1280, 384), "
                               "10% sparse Cholesky, mixed form, control variate per system",
                   "energy_every": args.energy_every, "timing": "wall clock, device-synchronised",
                   "kernel_tuning": tun},
        "fused_batch": {"value": res["fused"][0], "unit": METRIC,
                        "vhs_only": res["fused_vhs"][0], "chain_only": res["fused_chain"][0]},
        "independent_streams": {"value": res["independent"][0], "unit": METRIC},
        "serial": {"value": res["serial"][0], "unit": METRIC},
        "control_variate": cv,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    if args.config == "C5":
        run_c5(args, torch)
        return
    import torch.distributed as dist
    from datetime import timedelta
    import dataclasses
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    from miniafqmc_b200.synthetic import CONFIGS, make_system
    from miniafqmc_b200 import driver
    cfg = dataclasses.replace(CONFIGS[args.config], with_vakbl=False)
    if args.walkers:
        cfg = dataclasses.replace(cfg, nwalk=args.walkers)
    s = make_system(cfg)
    nw = cfg.nwalk
    comm = None
    if world > 1:
        def allreduce(vals):
            t = torch.tensor(vals, dtype=torch.float64, device="cuda")
            dist.all_reduce(t)
            return t.tolist()
        comm = driver.Comm(rank * nw, world * nw, allreduce,
                           driver.nccl_allreduce_device(torch, dist))

    head = Form(s, cfg, args, args.form, local, comm, torch)
    head.measure(record=False)
    # warm-up: W substeps, and for the control variate as many more as its first 2000
    # exact-exchange walker-steps take (walkers propagate in between, so the training set
    # spans the walkers' spread), until the estimator is on for the next measurement
    nwarm = args.warmup
    for st in range(nwarm):
        head.step(st, record=False)
    if head.mode == "cv":
        while not head.eng.cv_stats()["samples"] >= 2000 or nwarm % args.energy_every:
            head.step(nwarm, record=False)
            nwarm += 1
    with ClockSampler(local) as clk:
        ms, wall, _ = timed(head, args.steps, nwarm, torch, dist, world)
    # per-stage breakdown: the same number of further substeps, op by op with stage events
    _, _, stages = timed(head, args.steps, nwarm + args.steps, torch, dist, world, profile=True,
                         record=False)
    value = world * nw * args.steps / (ms * 1e-3)
    launches = int(sum(v[1] for v in stages.values()))

    # ---- end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        eng = head.eng
        K = args.steps
        xs = torch.empty((K, cfg.nchol, nw), dtype=torch.float64, pin_memory=True)
        xs.normal_(generator=torch.Generator().manual_seed(cfg.seed))
        wd = torch.empty((nw, 8, 2), dtype=torch.float64, pin_memory=True)
        xnp, wdnp = xs.numpy(), wd.numpy()
        eng.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k in range(K):
            st = nwarm + 2 * args.steps + k
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
                head.measure(record=False)
                if args.branch:
                    eng.population_control(cfg.seed, st + 1)
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
               "note": "per step: normals H2D (pinned) via afq_sigma_from, W_data D2H via "
                       "afq_get_walkers; energy every energy_every steps"}

    # ---- the plain FP64 form on the same steps and auxiliary fields (N=1)
    cmp = None
    if not args.no_fp64 and args.form != "fp64" and world == 1:
        ref = Form(s, cfg, args, "fp64", local, None, torch)
        ref.measure(record=False)
        for st in range(nwarm):
            ref.step(st, record=False)
        ms64, wall64, _ = timed(ref, args.steps, nwarm, torch, dist, world)
        _, _, stages64 = timed(ref, min(args.steps, 5), nwarm + args.steps, torch, dist, world,
                               profile=True, record=False)
        stages64 = {k: (v[0] * args.steps / min(args.steps, 5), v[1]) for k, v in stages64.items()}
        T_m, T_6 = ms * 1e-3, ms64 * 1e-3
        cmp = {
            "fp64_plain": {"value": nw * args.steps / T_6, "unit": METRIC,
                           "ms_per_step": ms64 / args.steps,
                           "stages_ms": {k: round(v[0], 3) for k, v in stages64.items()}},
            "speedup_vs_fp64_plain": T_6 / T_m,
            "energy": {},
        }
        # the same walkers measured by both forms: the mixed form's deterministic energy
        # error against FP64, and the control-variate estimate against exact exchange
        W, Wd = head.eng.get_walkers()
        ref.eng.set_walkers(W, Wd)
        ref.eng.calculate_mixed_density_matrix()
        e64 = ref.eng.calculate_energy("chol")
        head.eng.calculate_mixed_density_matrix()
        same = {"E_fp64_Ha": e64}
        if head.mode == "cv":
            ecv = head.eng.calculate_energy("cv")
            same["cv_minus_fp64_Ha"] = ecv - e64
            same["cv_sigma_Ha"] = float(np.sqrt(head.eng.cv_stats()["subset_var"]))
        emx = head.eng.calculate_energy("chol")
        same["mixed_exact_minus_fp64_Ha"] = emx - e64
        cmp["energy"]["same_walkers"] = same
        cmp["fp64_plain"]["kernel_tuning"] = ref.eng.tuning()
        cmp["fp64_plain"]["sparse_paths"] = ref.eng.sparse_paths()
        ref.eng.close()
        if head.mode == "cv" and args.acc_substeps > 0:
            cmp["energy"].update(accuracy_pass(s, cfg, args, local, torch))

    if rank != 0:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    # ---- roofline of the dominant stage
    peaks, src = measured_peaks()
    dom = max(stages, key=lambda k: stages[k][0])
    dom_ms, dom_launch = stages[dom]
    # calls of each stage in the profiled pass (substeps nwarm + K .. nwarm + 2K - 1): the
    # density matrix once per substep and once per measurement, the energy per measurement
    p0 = nwarm + args.steps
    nmeas = sum(1 for st in range(p0, p0 + args.steps) if (st + 1) % args.energy_every == 0)
    stage_calls = {"DM": args.steps + nmeas, "energy": max(nmeas, 1)}
    if args.form == "fp64":
        calls = stage_calls.get(dom, args.steps)
        peak = fp64_peak_tflops(torch)
        achieved = fp64_stage_flops(cfg, nw, dom) * calls / (dom_ms * 1e-3) / 1e12
        roof = {"kernel": dom, "bound": "fp64", "achieved": achieved, "peak": peak,
                "unit": "TFLOP/s", "frac": achieved / peak,
                "peak_source": "FP64 cuBLAS DGEMM 8192^3 measured in this run "
                               "(no FP64 entry in MEASURED_PEAKS.json)"}
    elif dom == "propagate":
        # algorithmic work and compulsory bytes of one substep's chain (8 launches): the
        # stage's 16 N^2 n complex multiply-adds per walker, against the bytes it cannot
        # avoid moving (V once, the P W operand in, W and its packed forms out); the larger
        # of the two lower bounds on the time names the roof
        preal = bool(np.all(np.asarray(s.Propg1).imag == 0))
        fl = prop_flops(cfg, nw) * args.steps
        by = prop_compulsory_bytes(cfg, nw, preal) * args.steps
        t_fl = fl / (peaks["bf16_tflops_sustained"] * 1e12)
        t_by = by / (peaks["hbm_gbs"] * 1e9)
        if t_fl >= t_by:
            achieved = fl / (dom_ms * 1e-3) / 1e12
            roof = {"kernel": "propagate (tcgen05 GEMM chain)", "bound": "tensor",
                    "achieved": achieved, "peak": peaks["bf16_tflops_sustained"],
                    "unit": "TFLOP/s", "frac": achieved / peaks["bf16_tflops_sustained"],
                    "peak_source": f"bf16_tflops_sustained, {src}"}
        else:
            achieved = by / (dom_ms * 1e-3) / 1e9
            roof = {"kernel": "propagate (tcgen05 GEMM chain)", "bound": "hbm",
                    "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                    "frac": achieved / peaks["hbm_gbs"], "peak_source": f"hbm_gbs, {src}"}
        roof["per_launch"] = "one substep's chain of 8 product launches"
        roof["algorithmic"] = {
            "flop_per_walker": prop_flops(cfg, 1), "bytes_per_walker": prop_compulsory_bytes(cfg, 1, preal),
            "t_flop_ms": t_fl * 1e3 / args.steps, "t_byte_ms": t_by * 1e3 / args.steps,
            "ms_measured": dom_ms / args.steps}
        roof["traffic_model"] = mixed_propagate_bytes(cfg, nw, preal=preal)
    else:
        calls = stage_calls.get(dom, args.steps)
        real_ops = bool(np.all(s.SpvnT.vals.imag == 0)) and (s.Lh is None or
                                                             bool(np.all(s.Lh.imag == 0)))
        sub = (nw + 7) // 8 if head.mode == "cv" else nw
        achieved = mixed_stage_flops(cfg, nw, dom, real_ops, sub) * calls / (dom_ms * 1e-3) / 1e12
        roof = {"kernel": dom, "bound": "tensor", "achieved": achieved,
                "peak": peaks["bf16_tflops_sustained"], "unit": "TFLOP/s",
                "frac": achieved / peaks["bf16_tflops_sustained"],
                "peak_source": f"bf16_tflops_sustained, {src}"}
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        tj = json.load(open(tpath)).get(f"{args.config}:{args.form}:{dom}")
        if tj is not None:   # DRAM bytes per launch unit, measured at a reduced walker count
            traffic = tj * nw / json.load(open(tpath)).get("_walkers", nw)
    roof.update({"traffic": traffic, "stage_ms": dom_ms, "launches": dom_launch,
                 "avg_launch_ms": dom_ms / max(dom_launch, 1)})
    if traffic is not None and dom == "propagate" and args.form != "fp64":
        roof["traffic_over_compulsory"] = traffic / (roof["algorithmic"]["bytes_per_walker"] * nw)

    cpu = None
    if not args.no_cpu and world == 1:
        threads = os.cpu_count() or 1
        r, info = cpu_rate(s, cfg, args, args.cpu_walkers or max(threads, 8), threads)
        cpu = {"value": r, "unit": METRIC, "cores": threads, "kind": "port", "sample": info["sample"]}

    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.form == "fp64" else "bf16 split/plain tensor-core + f64 LU/QR/weights",
        "data": "synthetic", "config": workload(cfg, args, nw),
        "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
        "clocks": clk.summary(), "stages_ms": {k: round(v[0], 3) for k, v in stages.items()},
    }
    if cmp:
        line.update(cmp)
    if head.mode == "cv":
        line["control_variate"] = head.eng.cv_stats()
    line["config"]["kernel_tuning"] = head.eng.tuning()
    if args.form == "fp64":
        line["config"]["sparse_paths"] = head.eng.sparse_paths()
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
