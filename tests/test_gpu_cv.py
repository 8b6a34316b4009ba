"""The learned control variate: the network's GPU forward/backward kernels against the
float64 oracle (oracle/mlp.py), its training, and the energy estimator built on it --
unbiased against the exact Cholesky energy and with a variance below that of plain
subsampling of the exact exchange (the method without the network)."""
import json
import os

import numpy as np
import pytest

from conftest import system
from oracle import mlp as M

pytestmark = pytest.mark.gpu
# with AFQ_TEST_RESULTS naming a directory, the measured figures are written there
OUT = (os.path.join(os.environ["AFQ_TEST_RESULTS"], "cv_results.json")
       if os.environ.get("AFQ_TEST_RESULTS") else None)


def test_mlp_forward_and_gradient_match_oracle():
    from miniafqmc_b200.afqmc import Mlp
    nin, H, B = 36, 256, 200
    net = Mlp(nin, H, capacity=512, seed=3)
    p = net.get_params()
    rng = np.random.default_rng(0)
    x = rng.normal(size=(B, nin)).astype(np.float32)
    t = rng.normal(size=B).astype(np.float32)
    y = net.forward(x)
    y_ref, _ = M.forward(p, x, nin, H)
    assert np.max(np.abs(y - y_ref)) / np.max(np.abs(y_ref)) < 1e-5
    g, loss = net.gradient(x, t)
    g_ref, loss_ref = M.gradient(p, x, t, nin, H)
    assert abs(loss - loss_ref) / loss_ref < 1e-5
    lay = M.layout(nin, H)
    for k, (a, b) in lay.items():
        err = np.max(np.abs(g[a:b] - g_ref[a:b])) / max(np.max(np.abs(g_ref[a:b])), 1e-12)
        assert err < 1e-4, (k, err)
    net.close()


def test_mlp_training_reduces_loss():
    from miniafqmc_b200.afqmc import Mlp
    nin, B = 36, 1024
    rng = np.random.default_rng(1)
    x = rng.normal(size=(B, nin)).astype(np.float32)
    t = (np.sin(x[:, 0]) + 0.5 * x[:, 1] * x[:, 2] - 0.3 * x[:, 3]).astype(np.float32)
    net = Mlp(nin, 256, capacity=B, seed=5)
    _, l0 = net.gradient(x, t)
    l1 = net.train(x, t, iters=300, lr=1e-3)
    assert l1 < 0.05 * l0
    net.close()


@pytest.mark.parametrize("opts", [{}, {"AFQ_CV_SAMPLING": "0"},
                                  {"AFQ_CV_RESIDUAL": "1", "AFQ_CV_QREFRESH": "5"},
                                  {"base": 1}])
def test_cv_energy_unbiased_with_variance_gain(opts, monkeypatch):
    """Default subset design (weight-proportional teeth over walkers ordered by the
    surrogate), the simple random sample, residual learning on a linearised exchange
    refreshed every five measurements (FP64 form), and the two-level surrogate of the
    mixed form (plain-bf16 exchange of every walker + learned residual): all unbiased,
    all with a variance gain."""
    from miniafqmc_b200.afqmc import AfqmcSys, AFQ_PREC_MIXED, AFQ_PREC_FP64
    opts = dict(opts)
    base = opts.pop("base", 0)
    for k, v in opts.items():
        monkeypatch.setenv(k, v)
    s = system("C1")
    nw = 256
    g = AfqmcSys(s, nw, precision=AFQ_PREC_MIXED if base else AFQ_PREC_FP64)
    g.cv_configure(hidden=256, lr=1e-3, seed=7, train_walker_steps=4 * nw, subset_den=8)
    if base:
        g.cv_set_base(1)
    diffs, gains, exact, htv = [], [], [], []
    st = 0
    for meas in range(40):
        for _ in range(2):
            g.substep(0, st, 5, graph=True)
            st += 1
        g.calculate_mixed_density_matrix()
        e_cv = g.calculate_energy("cv")
        stats = g.cv_stats()
        pred = g.copy_out("cv_pred")
        Wd_cv = g.get_walker_data()
        e_ex = g.calculate_energy("chol")
        ek = g.copy_out("energy_parts")[:, 2]
        Wd_ex = g.get_walker_data()
        if stats["active"]:
            # the subset's exact local energies are the exact evaluation's, walker by walker
            # (mixed form: the subset's exchange product may run another kernel variant
            # than the all-walker one, so the fp32 sums agree to rounding, not bitwise;
            # a walker outside the subset may then agree as closely by chance)
            tol = 1e-6 if base else 1e-9
            same = np.abs(Wd_cv[:, 0] - Wd_ex[:, 0]) <= tol * np.abs(Wd_ex[:, 0])
            if base:
                assert same.sum() >= stats["subset"], (same.sum(), stats["subset"])
            else:
                assert same.sum() == stats["subset"], (same.sum(), stats["subset"])
            diffs.append(e_cv - e_ex)
            om = Wd_cv[:, 1].real
            v_plain = np.var(om * ek, ddof=1)           # plain subsampling of exact E_K
            v_cv = np.var(om * (ek - pred), ddof=1)     # subsampling the residual
            gains.append(v_plain / v_cv)
            exact.append(e_ex)
            htv.append(stats["subset_var"])
        else:
            assert e_cv == pytest.approx(e_ex, rel=1e-6 if base else 1e-12)
    diffs = np.array(diffs)
    res = {"measurements_active": len(diffs), "mean_dE": float(diffs.mean()),
           "std_dE": float(diffs.std(ddof=1)), "median_variance_gain": float(np.median(gains)),
           "last_stats": stats, "E_exact_last": exact[-1],
           "predicted_std_dE": float(np.sqrt(np.mean(htv)))}
    if OUT is not None:
        os.makedirs(os.path.dirname(OUT), exist_ok=True)
        path = OUT if not base else OUT.replace(".json", "_base.json")
        with open(path, "w") as f:
            json.dump(res, f, indent=1)
    assert len(diffs) >= 20
    # unbiased: the mean deviation is within 4 standard errors of zero
    assert abs(diffs.mean()) < 4 * diffs.std(ddof=1) / np.sqrt(len(diffs)) + 1e-12
    # the trained surrogate removes most of the exchange variance of plain subsampling
    assert np.median(gains) > 3.0
    # the estimator's own sampling-variance estimate matches the observed scatter
    assert 0.4 < diffs.std(ddof=1) / np.sqrt(np.mean(htv)) < 2.5
    assert not stats["fallback"]
    g.close()
