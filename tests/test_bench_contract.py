"""The bench's JSON contract on the host (no GPU).

The reference arm (`bench.py --impl reference`: the FP64 CPU restatement of the reference
on the host cores) prints exactly one line with the contract's keys, and only rank 0
prints it.  The roofline's algorithmic models have their closed forms: the propagation
chain's HBM bytes (FP64 walkers out, each bf16 operand read once, the fp32 Taylor sum
read and written, the new walkers' packed forms written by the last product) and the
tensor-core FLOPs of the vHS stage."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

CONTRACT_KEYS = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better",
                 "scaling", "vs_baseline", "dtype", "data", "config")


def run_bench(args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT,
                          capture_output=True, text=True, timeout=600, env=e)


def test_reference_arm_prints_one_contract_line():
    out = run_bench(["--impl", "reference", "--config", "C1", "--steps", "1", "--warmup", "3",
                     "--cpu-walkers", "4"])
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in CONTRACT_KEYS:
        assert k in d, k
    assert d["impl"] == "reference" and d["metric"] == "walker-steps/s"
    assert d["value"] > 0 and d["higher_is_better"] is True and d["steps"] == 1
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["kind"] == "port"
    assert d["cpu_baseline"]["cores"] >= 1 and "4 walkers" in d["cpu_baseline"]["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert d["config"]["workload"].startswith("C1:")


def test_reference_arm_other_ranks_print_nothing():
    out = run_bench(["--impl", "reference", "--config", "C1", "--steps", "1", "--warmup", "3",
                     "--cpu-walkers", "4"], env={"RANK": "1"})
    assert out.returncode == 0 and out.stdout.strip() == ""


def test_propagation_byte_model():
    sys.path.insert(0, ROOT)
    import bench
    from miniafqmc_b200.synthetic import CONFIGS
    cfg = CONFIGS["C4"]
    N, n, nw = cfg.nmo, cfg.nel, 1024
    W64 = nw * N * 2 * n * 16                  # FP64 walkers [nw][2][N][n]
    F = nw * 4 * n * 2 * N * 2                 # one bf16 part of a complex-as-real B operand
    Fp = F // 2                                # real Propg1: K = N
    V = nw * N * 2 * N * 2                     # one bf16 part of the V operand
    S = nw * N * 2 * n * 8                     # fp32 Taylor sum
    pw = 2 * Fp + S + 2 * F                    # S = P W
    t1 = 2 * V + 2 * F + 2 * S + F             # first Taylor term (split V and B)
    tk = V + F + 2 * S + F                     # terms 2-5 (plain bf16)
    t6 = V + F + 2 * S + 2 * Fp                # term 6 forms the P S operand
    ps = 2 * Fp + W64 + F + 2 * Fp             # W = P S + T1 operand + next P W operand
    want = pw + t1 + 4 * tk + t6 + ps
    assert bench.mixed_propagate_bytes(cfg, nw) == pytest.approx(want, rel=1e-15)
    assert want == pytest.approx(14.4955e9, rel=1e-4)
    # every term scales with the walker count
    assert bench.mixed_propagate_bytes(cfg, 2 * nw) == pytest.approx(2 * want, rel=1e-15)
    # a complex Propg1: the four P-product operands (hi + lo each) have K = 2N
    cplx = want + 4 * 2 * (F - Fp)
    assert bench.mixed_propagate_bytes(cfg, nw, preal=False) == pytest.approx(cplx, rel=1e-15)


def test_vhs_flop_model():
    sys.path.insert(0, ROOT)
    import bench
    from miniafqmc_b200.synthetic import CONFIGS
    cfg = CONFIGS["C4"]
    N, nc, nw = cfg.nmo, cfg.nchol, 1024
    # real Spvn x complex X over the N(N+1)/2 symmetric orbital pairs: 4 FLOP each
    assert bench.mixed_stage_flops(cfg, nw, "vHS") == 4.0 * nw * (N * (N + 1) // 2) * nc


def test_propagation_roofline_models():
    """Algorithmic work of one propagation: 16 N^2 n complex multiply-adds per walker at
    Taylor order 6; compulsory bytes: V once (hi + lo), the packed P W operand in, the FP64
    walkers and their two packed forms out.  At C4 the FLOP bound is the larger one."""
    sys.path.insert(0, ROOT)
    import bench
    from miniafqmc_b200.synthetic import CONFIGS
    cfg = CONFIGS["C4"]
    N, n = cfg.nmo, cfg.nel
    assert bench.prop_flops(cfg, 1) == 8.0 * 16 * N * N * n
    V, Fp, T1, W64 = 2 * N * 2 * N * 2, 4 * n * N * 2, 2 * n * 2 * N * 4, N * 2 * n * 16
    assert bench.prop_compulsory_bytes(cfg, 1) == V + 2 * Fp + W64 + T1 + 2 * Fp
    assert bench.prop_compulsory_bytes(cfg, 1) < bench.mixed_propagate_bytes(cfg, 1) / 5
    assert bench.prop_flops(cfg, 1) / 1314.4e12 > bench.prop_compulsory_bytes(cfg, 1) / 6545.6e9


def test_blocking_sigma():
    """Blocking analysis (Flyvbjerg-Petersen): white noise gives the naive standard error;
    an AR(1) series with correlation time tau gives about sqrt(2 tau) times more."""
    sys.path.insert(0, ROOT)
    import bench
    import numpy as np
    rng = np.random.default_rng(1)
    x = rng.normal(size=4096)
    s, lev = bench.blocking_sigma(x)
    assert len(lev) == 10 and abs(lev[0] - x.std(ddof=1) / 64) < 1e-12
    assert 0.8 < s / lev[0] < 1.3
    phi = 0.9                                  # tau_int = (1 + phi) / (1 - phi) / 2 = 9.5
    y = np.zeros(8192)
    for i in range(1, len(y)):
        y[i] = phi * y[i - 1] + rng.normal()
    s, lev = bench.blocking_sigma(y)
    assert 3.0 < s / lev[0] < 5.5             # sqrt(2 tau_int) = 4.36


def test_accuracy_pass_report_structure(monkeypatch):
    """The energy-accuracy pass's bookkeeping on the host, with a stand-in for the GPU
    walker sets: four trajectories (both control-variate settings, exact exchange, FP64),
    the two shadow estimators on the FP64 trajectory's walkers, and the keys of the
    report (|dE| on identical fields with its z-score, the identical-walker figures, the
    other setting's summary and the energy error per wall-second)."""
    import types
    import numpy as np
    import bench

    class FakeTorchEvent:
        t = 0.0

        def __init__(self, **kw):
            self.t = 0.0

        def record(self, stream=None):
            FakeTorchEvent.t += 1.0
            self.t = FakeTorchEvent.t

        def elapsed_time(self, other):
            return 1000.0 * (other.t - self.t)

    torch = types.SimpleNamespace(cuda=types.SimpleNamespace(
        Event=FakeTorchEvent, synchronize=lambda: None))

    class FakeEng:
        def __init__(self, name, base):
            self.name, self.base, self.k = name, base, 0
            self.rng = np.random.default_rng(hash((name, base)) % 2**32)

        def synchronize(self):
            pass

        def copy_walkers_from(self, other):
            self.k = other.k

        def calculate_mixed_density_matrix(self):
            pass

        def calculate_energy(self, mode):
            e = -300.0 + 0.1 * np.sin(self.k)
            if mode == "cv":
                e += (1e-5 if self.base else 1e-3) * self.rng.normal()
            return float(e)

        def cv_stats(self):
            return {"subset_var": 1e-6, "active": True}

        def close(self):
            pass

    class FakeForm:
        def __init__(self, system, cfg, args, form, device, comm, torch, cv_base=None):
            self.form = form
            self.mode = "cv" if form == "mixed-cv" else "chol"
            self.cv_base = args.cv_base if cv_base is None else cv_base
            self.eng = FakeEng(form, self.cv_base)
            self.stream = None
            self.energies, self.cvvar = [], []

        def measure(self, record=True):
            E = self.eng.calculate_energy(self.mode)
            if record:
                self.energies.append(E)
                if self.mode == "cv":
                    self.cvvar.append(1e-6)
            return E

        def step(self, st, record=True, graph=True):
            self.eng.k = st + 1
            if (st + 1) % 5 == 0:
                self.measure(record)

    monkeypatch.setattr(bench, "Form", FakeForm)
    args = types.SimpleNamespace(acc_substeps=100, acc_equil=20, energy_every=5, cv_base=0)
    out = bench.accuracy_pass(None, None, args, 0, torch)
    assert set(out["forms"]) == {"mixed-cv", "mixed-cv-two-level", "mixed", "fp64"}
    assert set(out["same_walkers_along_fp64_trajectory"]) == {"cv", "cv_two_level", "exact"}
    for k in ("abs_dE_Ha", "abs_dE_sigma_Ha", "abs_dE_z", "same_walkers_abs_dE_Ha",
              "same_walkers_abs_dE_sigma_Ha", "abs_dE_deterministic_Ha"):
        assert np.isfinite(out[k]), k
    assert out["other_control_variate"]["form"] == "cv_two_level"
    assert out["forms"]["mixed-cv-two-level"]["low_precision_base"] is True
    assert out["err_per_wall_s"]["fp64_over_form"] > 0
    json.dumps(out)
