"""Cross-checks of the FP64 oracle against an independent numpy restatement of the
reference's formulas (Appendix-style, written from afqmc_sys.hpp / vHS.hpp /
miniafqmc_base.cpp), plus the energy identity and the half-rotation.

The Householder restatement here is the algorithm the GPU re-orthogonalisation kernel
runs; checking it against LAPACK's zgelqf + zunglq (inside the oracle) pins its
conventions on the CPU."""
import numpy as np
import pytest

from conftest import system, tiny_system
from oracle import oracle as O


def np_dm(sysm, W):
    nw = W.shape[0]
    N, n = sysm.N, sysm.n
    Gc = np.zeros((2 * n * N, nw), np.complex128)
    ov = np.zeros((nw, 2), np.complex128)
    for w in range(nw):
        for s in range(2):
            T1 = W[w, s].T @ sysm.trial[s]
            ov[w, s] = np.linalg.det(T1)
            Gc[s * n * N:(s + 1) * n * N, w] = (np.linalg.inv(T1) @ W[w, s].T).ravel()
    return Gc, ov


def np_propagate(sysm, W, vHS, order=6):
    N = sysm.N
    W = W.copy()
    for w in range(W.shape[0]):
        V = vHS[:, w].reshape(N, N)
        for s in range(2):
            S = sysm.Propg1 @ W[w, s]
            T = S.copy()
            for k in range(1, order + 1):
                T = (1j / k) * (V @ T)
                S = S + T
            W[w, s] = sysm.Propg1 @ S
    return W


def householder_lq(Wm):
    """zgelqf + zunglq of the row-major N x n block as the GPU kernel computes it:
    QR of conj(W) with zlarfg reflectors, Q formed backwards, W <- conj(Q)."""
    B = np.conj(Wm).astype(np.complex128).copy()
    N, n = B.shape
    taus = np.zeros(n, np.complex128)
    for j in range(n):
        alpha = B[j, j]
        xn2 = np.sum(np.abs(B[j + 1:, j]) ** 2)
        if xn2 == 0.0 and alpha.imag == 0.0:
            continue
        beta = -np.copysign(np.sqrt(abs(alpha) ** 2 + xn2), alpha.real)
        tau = complex((beta - alpha.real) / beta, -alpha.imag / beta)
        B[j + 1:, j] /= (alpha - beta)
        B[j, j] = beta
        v = np.concatenate([[1.0], B[j + 1:, j]])
        s = np.conj(v) @ B[j:, j + 1:]
        B[j:, j + 1:] -= np.conj(tau) * np.outer(v, s)
        taus[j] = tau
    for i in reversed(range(n)):
        tau = taus[i]
        if i < n - 1:
            v = np.concatenate([[1.0], B[i + 1:, i]])
            s = np.conj(v) @ B[i:, i + 1:]
            B[i:, i + 1:] -= tau * np.outer(v, s)
        B[i + 1:, i] *= -tau
        B[i, i] = 1.0 - tau
        B[:i, i] = 0.0
    return np.conj(B)


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("cplx", [False, True])
def test_oracle_substep_matches_numpy(cplx):
    s = tiny_system(complex_trial=cplx, complex_chol=cplx)
    nw = 4
    o = O.Oracle(s, nw)
    W0, Wd0 = s.initial_walkers(nw)
    rng = np.random.default_rng(3)
    W0 = W0 + 0.05 * (rng.normal(size=W0.shape) + 1j * rng.normal(size=W0.shape))
    o.set_walkers(W0, Wd0)
    o.calculate_mixed_density_matrix()
    Gc, ov = np_dm(s, W0)
    assert rel(o.copy_out("Gc"), Gc) < 1e-12
    _, Wd = o.get_walkers()
    assert rel(Wd[:, 2:4], ov) < 1e-12
    o.get_vbias()
    vb = s.SpvnT.todense() @ Gc
    assert rel(o.copy_out("vbias"), vb) < 1e-12
    o.sigma(5, 2)
    x = o.copy_out("xraw")
    X = x + 1j * vb
    assert rel(o.copy_out("X"), X) < 1e-12
    hw = -(1j * vb * (x + 0.5j * vb)).sum(axis=0)
    assert rel(o.copy_out("hybridW"), hw) < 1e-12
    o.get_vHS()
    vHS = s.Spvn.todense() @ X
    assert rel(o.copy_out("vHS"), vHS) < 1e-12
    o.propagate()
    W1 = np_propagate(s, W0, vHS)
    W, _ = o.get_walkers()
    assert rel(W, W1) < 1e-12


def test_oracle_weights_match_driver_formula():
    s = tiny_system()
    nw = 4
    o = O.Oracle(s, nw)
    o.calculate_mixed_density_matrix()
    o.get_vbias()
    o.sigma(1, 0)
    o.get_vHS()
    o.propagate()
    _, Wd_before = o.get_walkers()
    o.calculate_overlaps(save_old=True)
    o.eshift = -1.5
    o.update_weights()
    _, Wd = o.get_walkers()
    hw = o.copy_out("hybridW")
    dt = s.cfg.dt
    ratio = Wd[:, 2] * Wd[:, 3] / (Wd_before[:, 2] * Wd_before[:, 3])
    e4 = -(hw + np.log(ratio)) / dt
    scale = np.maximum(0.0, np.cos(np.angle(ratio)))
    w = scale * np.exp(-dt * (0.5 * (e4.real + Wd_before[:, 4].real) + 1.5))
    np.testing.assert_allclose(Wd[:, 4], e4, rtol=1e-12)
    np.testing.assert_allclose(Wd[:, 1].real, w, rtol=1e-12)
    assert o.eshift == pytest.approx(e4.real.mean(), rel=1e-12)


@pytest.mark.parametrize("shape", [(12, 3), (40, 7), (64, 16)])
def test_householder_restatement_matches_lapack_lq(shape):
    N, n = shape
    rng = np.random.default_rng(N)
    from miniafqmc_b200.synthetic import Config, make_system
    s = make_system(Config(N, n, 4, 0.3, 1, nwalk=2))
    W = rng.normal(size=(2, 2, N, n)) + 1j * rng.normal(size=(2, 2, N, n))
    o = O.Oracle(s, 2)
    o.set_walkers(W, np.zeros((2, 8), np.complex128))
    o.orthogonalize()
    Wq, _ = o.get_walkers()
    for w in range(2):
        for sp in range(2):
            Q = householder_lq(W[w, sp])
            assert rel(Q, Wq[w, sp]) < 1e-12
            np.testing.assert_allclose(Q.conj().T @ Q, np.eye(n), atol=1e-12)


@pytest.mark.parametrize("cplx", [False, True])
def test_energy_vakbl_equals_cholesky(cplx):
    s = tiny_system(complex_trial=cplx, complex_chol=cplx)
    o = O.Oracle(s, 4)
    rng = np.random.default_rng(1)
    W, Wd = s.initial_walkers(4)
    W = W + 0.1 * (rng.normal(size=W.shape) + 1j * rng.normal(size=W.shape))
    Wd[:, 1] = rng.uniform(0.5, 1.5, 4)
    o.set_walkers(W, Wd)
    o.calculate_mixed_density_matrix()
    e_v = o.calculate_energy("vakbl")
    _, Wv = o.get_walkers()
    e_c = o.calculate_energy("chol")
    _, Wc = o.get_walkers()
    assert e_v == pytest.approx(e_c, rel=1e-12)
    np.testing.assert_allclose(Wv[:, 0], Wc[:, 0], rtol=1e-11)


def test_halfrotate_restatement_matches_generator():
    s = system("C1")
    ri, ci, v = O.halfrotate(s)
    np.testing.assert_array_equal(ri, s.SpvnT.rowIndex)
    np.testing.assert_array_equal(ci, s.SpvnT.cols)
    assert np.max(np.abs(v - s.SpvnT.vals)) < 1e-15


def test_trajectory_is_deterministic_and_threads_agree():
    s = tiny_system()
    res = []
    for threads in (1, 4):
        o = O.Oracle(s, 6, threads=threads)
        for st in range(6):
            o.substep(11, st, 3)
        res.append(o.get_walkers())
    np.testing.assert_array_equal(res[0][0], res[1][0])
    np.testing.assert_array_equal(res[0][1], res[1][1])


def test_mlp_oracle_gradient_by_finite_differences():
    """Pins the network oracle: analytic gradient vs central differences (float64,
    unrounded weights)."""
    from oracle import mlp as M
    rng = np.random.default_rng(0)
    nin, H, B = 5, 32, 7
    P = M.layout(nin, H)["b3"][1]
    p = rng.normal(scale=0.3, size=P)
    x = rng.normal(size=(B, nin))
    t = rng.normal(size=B)
    g, _ = M.gradient(p, x, t, nin, H, round_weights=False)
    loss = lambda q: 0.5 * np.mean((M.forward(q, x, nin, H, round_weights=False)[0] - t) ** 2)
    for i in rng.choice(P, 40, replace=False):
        e = np.zeros(P)
        e[i] = 1e-6
        fd = (loss(p + e) - loss(p - e)) / 2e-6
        assert abs(fd - g[i]) < 1e-6 + 1e-5 * abs(g[i])


def test_bf16_rounding_matches_torch():
    import torch
    from oracle import mlp as M
    x = np.random.default_rng(1).normal(size=10000).astype(np.float32) * 100
    ref = torch.from_numpy(x).bfloat16().float().numpy()
    np.testing.assert_array_equal(M.bf16(x), ref)


@pytest.mark.parametrize("cplx", [False, True])
def test_oracle_full_g_path_matches_numpy(cplx):
    """The oracle's transposed_Spvn == false branch: G_s = trial_s T1^-1 W_s^T
    (mixed_density_matrix.hpp:96-99) and vbias = T(Spvn) G_alpha + T(Spvn) G_beta
    (vbias.hpp:66-81), against numpy; and equal to the compact path's vbias without the
    half-rotation cutoff (SpvnT built from the same Spvn and trial)."""
    s = tiny_system(complex_trial=cplx, complex_chol=cplx)
    nw = 4
    N, n = s.N, s.n
    o = O.Oracle(s, nw)
    W0, Wd0 = s.initial_walkers(nw)
    rng = np.random.default_rng(5)
    W0 = W0 + 0.05 * (rng.normal(size=W0.shape) + 1j * rng.normal(size=W0.shape))
    o.set_walkers(W0, Wd0)
    o.calculate_mixed_density_matrix_full()
    G = np.zeros((2 * N * N, nw), np.complex128)
    for w in range(nw):
        for sp in range(2):
            T1 = W0[w, sp].T @ s.trial[sp]
            G[sp * N * N:(sp + 1) * N * N, w] = (s.trial[sp] @ np.linalg.inv(T1) @ W0[w, sp].T).ravel()
    assert rel(o.copy_out("G_full"), G) < 1e-12
    o.get_vbias_full()
    Sp = s.Spvn.todense()
    vb = Sp.T @ G[:N * N] + Sp.T @ G[N * N:]
    assert rel(o.copy_out("vbias"), vb) < 1e-12
    Gc, _ = np_dm(s, W0)
    Lh = s.Lh.reshape(s.nchol, 2 * n * N) * np.sqrt(s.cfg.dt)   # no cutoff
    assert rel(np.asarray(Lh @ Gc), vb) < 1e-12


def test_comb_restatement_properties():
    """The oracle's comb (the GPU test's reference): every copy's parent has positive weight, parents
    appear in walker order, and walker i gets floor or ceil of nw w_i / T copies."""
    from oracle.oracle import comb
    rng = np.random.default_rng(2)
    nw = 200
    W = rng.normal(size=(nw, 2, 3, 2))
    Wd = np.zeros((nw, 8), np.complex128)
    Wd[:, 1] = rng.lognormal(0.0, 1.0, nw)
    Wd[::5, 1] = 0.0
    for seed, step in ((1, 0), (1, 1), (9, 77)):
        Wn, Wdn, idx = comb(W, Wd, seed, step)
        w = np.maximum(Wd[:, 1].real, 0)
        assert np.all(w[idx] > 0) and np.all(np.diff(idx) >= 0)
        counts = np.bincount(idx, minlength=nw)
        expect = nw * w / w.sum()
        assert np.all(counts >= np.floor(expect) - 1e-9) and np.all(counts <= np.ceil(expect) + 1e-9)
        assert np.allclose(Wdn[:, 1].real, w.sum() / nw)
