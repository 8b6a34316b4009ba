"""The mixed-precision (tcgen05) form against the FP64 form on identical inputs.

Stage tolerances (relative to the largest magnitude of the quantity; overlaps relative
per walker):
  split bf16 (hi*hi + hi*lo + lo*hi) stages: 1e-4    plain bf16 stages: 2e-2
  overlaps: 5e-6 * n (the determinant of the n x n T1 sums the relative errors of its n
  pivots: 2-5e-5 measured at n = 16 and 32, 1.6e-4 at n = 64)
Trajectory: per-step mixed energy within 1e-4 relative of the FP64 energy on the same
auxiliary fields.  With AFQ_TEST_RESULTS naming a directory, the measured errors are also
written there as JSON (mixed_errors.json)."""
import json
import os

import numpy as np
import pytest

from conftest import system

pytestmark = pytest.mark.gpu
OUT = (os.path.join(os.environ["AFQ_TEST_RESULTS"], "mixed_errors.json")
       if os.environ.get("AFQ_TEST_RESULTS") else None)
ERRS = {}


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def record(key, val):
    ERRS[key] = val
    if OUT is None:
        return
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    with open(OUT, "w") as f:
        json.dump(ERRS, f, indent=1)


def pair(s, nw, walkers):
    from miniafqmc_b200.afqmc import AfqmcSys, AFQ_PREC_FP64, AFQ_PREC_MIXED
    d = AfqmcSys(s, nw, precision=AFQ_PREC_FP64, walkers=walkers)
    m = AfqmcSys(s, nw, precision=AFQ_PREC_MIXED, walkers=walkers)
    return d, m


def perturbed(s, nw, seed=0, amp=0.05):
    rng = np.random.default_rng(seed)
    W, Wd = s.initial_walkers(nw)
    W = W + amp * (rng.normal(size=W.shape) + 1j * rng.normal(size=W.shape))
    Wd[:, 1] = rng.uniform(0.5, 1.5, nw)
    return W, Wd


@pytest.mark.parametrize("name,kw,nw", [("C1", {}, 16),
                                        ("C1", dict(complex_trial=True, complex_chol=True,
                                                    nchol=96, seed=5), 16),
                                        ("C2", dict(with_vakbl=False), 64),
                                        ("C3", {}, 64)])
def test_mixed_stages(name, kw, nw):
    s = system(name, **kw)
    tag = name + ("c" if kw.get("complex_chol") else "")
    d, m = pair(s, nw, perturbed(s, nw))
    for e in (d, m):
        e.calculate_mixed_density_matrix()
        e.get_vbias()
    eg = rel(m.copy_out("Gc"), d.copy_out("Gc"))
    od, om = d.get_walker_data()[:, 2:4], m.get_walker_data()[:, 2:4]
    eo = float(np.max(np.abs(om - od) / np.abs(od)))
    ev = rel(m.copy_out("vbias"), d.copy_out("vbias"))
    for e in (d, m):
        e.sigma(3, 1)
        e.get_vHS()
    eh = rel(m.copy_out("vHS"), d.copy_out("vHS"))
    for e in (d, m):
        e.propagate()
    ew = rel(m.get_walkers()[0], d.get_walkers()[0])
    for e in (d, m):
        e.calculate_mixed_density_matrix()
    ed, em = d.calculate_energy("chol"), m.calculate_energy("chol")
    pd, pm = d.copy_out("energy_parts"), m.copy_out("energy_parts")
    m.synchronize()
    res = {"Gc": eg, "overlap": eo, "vbias": ev, "vHS": eh, "W_after_propagate": ew,
           "E": abs(em - ed) / abs(ed),
           "E1": rel(pm[:, 0], pd[:, 0]), "EJ": rel(pm[:, 1], pd[:, 1]), "EK": rel(pm[:, 2], pd[:, 2]),
           "E_abs_Ha": abs(em - ed)}
    record(f"stages_{tag}", res)
    assert eg < 1e-4 and eo < 5e-6 * s.n and ev < 1e-4 and eh < 1e-4
    assert ew < 2e-2
    assert res["EJ"] < 1e-4 and res["EK"] < 1e-4
    d.close()
    m.close()


@pytest.mark.parametrize("name,nw,nsub", [("C1", 16, 20), ("C3", 64, 10)])
def test_mixed_trajectory(name, nw, nsub):
    """Graph substeps of both forms on the same fields.  C3 (Spvn 30% nonzero, 64+64
    electrons) runs 64 of its 512 walkers: each walker's trajectory depends on the others
    only through the weights' energy shift."""
    s = system(name)
    d, m = pair(s, nw, None)
    dE = []
    for e in (d, m):
        e.calculate_mixed_density_matrix()
    for st in range(nsub):
        for e in (d, m):
            e.substep(0, st, 5, graph=True)
            e.calculate_mixed_density_matrix()
        ed, em = d.calculate_energy("chol"), m.calculate_energy("chol")
        dE.append(abs(em - ed))
    m.synchronize()
    record(f"trajectory_{name}", {"max_abs_dE_Ha": max(dE), "dE_per_step": dE, "E_last": ed})
    assert max(dE) / abs(ed) < 1e-4
    d.close()
    m.close()


def test_cholqr2_ortho_matches_householder_up_to_signs():
    """The mixed form re-orthogonalises with CholeskyQR2: same column space as the FP64
    form's LAPACK-convention Householder QR, columns equal up to +-1, so the density
    matrix is identical and overlaps agree in magnitude."""
    s = system("C1", complex_trial=True, complex_chol=True, nchol=96, seed=5)
    nw = 8
    d, m = pair(s, nw, perturbed(s, nw, amp=0.3))
    for e in (d, m):
        e.orthogonalize()
        e.calculate_mixed_density_matrix()
    Wd_, Wm = d.get_walkers()[0], m.get_walkers()[0]
    for w in range(nw):
        for sp in range(2):
            M = Wm[w, sp].conj().T @ Wd_[w, sp]
            assert np.max(np.abs(np.abs(M) - np.eye(s.n))) < 1e-11
    # the mixed form's density matrix and overlaps are split-bf16 tensor-core products
    assert rel(m.copy_out("Gc"), d.copy_out("Gc")) < 1e-4
    od, om = d.get_walker_data()[:, 2:4], m.get_walker_data()[:, 2:4]
    assert rel(np.abs(om), np.abs(od)) < 1e-4
    d.close()
    m.close()


def test_fp16_split_g_products(monkeypatch):
    """The fp16 hi/lo form (power-of-two scaled operands) of the vbias, Coulomb and
    exchange products agrees with the FP64 form like the bf16 split form (1e-4)."""
    monkeypatch.setenv("AFQ_MIXED_PREC", "vbias=2,ej=2,ek=2")
    s = system("C1")
    nw = 16
    d, m = pair(s, nw, perturbed(s, nw))
    for e in (d, m):
        e.calculate_mixed_density_matrix()
        e.get_vbias()
    ev = rel(m.copy_out("vbias"), d.copy_out("vbias"))
    ed, em = d.calculate_energy("chol"), m.calculate_energy("chol")
    pd, pm = d.copy_out("energy_parts"), m.copy_out("energy_parts")
    m.synchronize()
    res = {"vbias": ev, "E": abs(em - ed) / abs(ed), "EJ": rel(pm[:, 1], pd[:, 1]),
           "EK": rel(pm[:, 2], pd[:, 2])}
    record("fp16_g_C1", res)
    assert ev < 1e-4 and res["EJ"] < 1e-4 and res["EK"] < 1e-4 and res["E"] < 1e-5
    d.close()
    m.close()


@pytest.mark.parametrize("spread", [0.0, 3.0])
def test_cholqr_orthonormal_with_one_or_two_passes(spread):
    """Mixed-form re-orthogonalisation: well-conditioned walkers take one Cholesky-QR
    pass, ill-conditioned ones (columns scaled over three decades, kappa ~ 1e3) take two;
    both end orthonormal to 1e-11 with the same column space as before."""
    from miniafqmc_b200.afqmc import AfqmcSys, AFQ_PREC_MIXED
    s = system("C1")
    nw = 8
    W, Wd = perturbed(s, nw, amp=0.05)
    W = W * (10.0 ** (spread * np.arange(s.n) / s.n))[None, None, None, :]
    m = AfqmcSys(s, nw, precision=AFQ_PREC_MIXED, walkers=(W, Wd))
    m.orthogonalize()
    Wo = m.get_walkers()[0]
    for w in range(nw):
        for sp in range(2):
            Q = Wo[w, sp]
            assert np.max(np.abs(Q.conj().T @ Q - np.eye(s.n))) < 1e-11
            # same column space: W = Q (Q^H W)
            X = W[w, sp]
            assert np.max(np.abs(Q @ (Q.conj().T @ X) - X)) < 1e-10 * np.max(np.abs(X))
    m.close()


@pytest.mark.parametrize("name,kw,nw", [("C1", {}, 16), ("C2", dict(with_vakbl=False), 32)])
def test_packed_forms_equal_packing_from_w(name, kw, nw):
    """The last propagation product writes the new walkers' T1 and P W operands itself,
    and the orthogonalisation repacks them; population control and set_walkers mark them
    stale.  Overlaps, density matrix and the next propagation from those forms are bit for
    bit the ones of a handle given the same walkers (which packs them from W)."""
    from miniafqmc_b200.afqmc import AfqmcSys, AFQ_PREC_MIXED
    s = system(name, **kw)
    e = AfqmcSys(s, nw, precision=AFQ_PREC_MIXED, walkers=perturbed(s, nw, seed=4))

    def step(x, k):
        x.calculate_mixed_density_matrix()
        x.get_vbias()
        x.sigma(7, k)
        x.get_vHS()
        x.propagate()

    step(e, 1)
    for k, change in enumerate(("none", "ortho", "population")):
        if change == "ortho":
            e.orthogonalize()
        elif change == "population":
            e.population_control(11, k)
        f = AfqmcSys(s, nw, precision=AFQ_PREC_MIXED, walkers=e.get_walkers())
        for x in (e, f):
            x.calculate_overlaps()
        assert np.array_equal(e.get_walker_data(), f.get_walker_data()), change
        for x in (e, f):
            step(x, 2 + k)
        assert np.array_equal(e.copy_out("Gc"), f.copy_out("Gc")), change
        We, Wf = e.get_walkers(), f.get_walkers()
        assert np.array_equal(We[0], Wf[0]) and np.array_equal(We[1], Wf[1]), change
        f.close()
    e.close()


def test_copy_walkers_between_forms():
    """afq_copy_walkers: the mixed form measures the FP64 form's walkers after a device
    copy (energy within the absolute 1e-4 Ha bar of the FP64 energy of the same walkers);
    handles of another shape are refused."""
    from miniafqmc_b200.afqmc import AfqmcSys, AfqmcError, AFQ_PREC_FP64, AFQ_PREC_MIXED
    s = system("C1")
    nw = 16
    d = AfqmcSys(s, nw, precision=AFQ_PREC_FP64)
    m = AfqmcSys(s, nw, precision=AFQ_PREC_MIXED)
    d.calculate_mixed_density_matrix()
    for st in range(7):
        d.substep(2, st, 5, graph=True)
    m.copy_walkers_from(d)
    assert np.array_equal(m.get_walkers()[0], d.get_walkers()[0])
    assert np.array_equal(m.get_walker_data(), d.get_walker_data())
    for e in (d, m):
        e.calculate_mixed_density_matrix()
    ed, em = d.calculate_energy("chol"), m.calculate_energy("chol")
    assert abs(em - ed) < 1e-4
    m.substep(2, 7, 5, graph=True)         # the copy leaves the mixed handle usable
    assert np.all(np.isfinite(m.get_walker_data()))
    other = AfqmcSys(s, 8, precision=AFQ_PREC_MIXED)
    with pytest.raises(AfqmcError):
        other.copy_walkers_from(d)
    for e in (d, m, other):
        e.close()


def test_vhs_tile_epilogue_matches_rowwise(monkeypatch):
    """The symmetric vHS product's epilogues -- row-wise (each lane its walker's entries),
    through the fp32 tile in shared memory (16-byte rows, mirrored block included), and
    the same with two CTAs per SM staging the tile in two halves -- write the same V bit for
    bit: the same MMAs and the same bf16 rounding.  With 64-byte K slabs (choice 3) the MMA
    order over K changes: fp32 rounding over K = nchol, well inside the product's own error
    against FP64 (about 1e-5): 1.5e-5 relative (measured 6e-6).
    80 walkers: the second M tile holds 16 walkers and 96 empty rows."""
    from miniafqmc_b200.afqmc import AfqmcSys, AFQ_PREC_MIXED
    monkeypatch.delenv("AFQ_TUNE", raising=False)
    s = system("C2", with_vakbl=False)
    nw = 80
    wk = perturbed(s, nw)
    out = {}
    for ve in ("0", "1", "2", "3"):
        monkeypatch.setenv("AFQ_VHS_EPI", ve)
        m = AfqmcSys(s, nw, precision=AFQ_PREC_MIXED, walkers=wk, use_vakbl=False)
        assert m.tuning()["vhs_epilogue"]["tile"] == int(ve)
        m.calculate_mixed_density_matrix()
        m.get_vbias()
        m.sigma(3, 1)
        m.get_vHS()
        out[ve] = m.copy_out("vHS")
        m.close()
    assert np.array_equal(out["0"], out["1"])
    assert np.array_equal(out["0"], out["2"])
    # 64-byte K slabs: the same products, another fp32 summation order
    assert rel(out["3"], out["0"]) < 1.5e-5

