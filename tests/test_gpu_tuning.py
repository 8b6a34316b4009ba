"""Kernel autotuning of the mixed-precision products (no reference counterpart).

afq_set_hamiltonian times the persistent and the per-tile tensor-core kernel of each
product site (and the split-K slice count of vbias / Coulomb) on the handle's shapes and
keeps the fastest.  Both kernels run the same MMA sequence per tile, so forcing one or the
other (AFQ_TUNE=1 / 2) gives the same density matrix, vbias, vHS and walkers to 1e-12
relative (forcing a kernel also keeps the default slice count); the split-K products
promote their accumulator every few K slabs and run on the persistent kernel only; the
exchange of the per-tile kernel keeps one accumulation chain over K (1e-5 relative on
E_K against the promoted persistent one).  The timed choice
is cached per shape, and in AFQ_TUNE_CACHE when set."""
import numpy as np
import pytest

from conftest import system

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def run_step(s, nw, walkers):
    """One step of the stage sequence, returning the intermediate arrays."""
    from miniafqmc_b200.afqmc import AfqmcSys, AFQ_PREC_MIXED
    e = AfqmcSys(s, nw, precision=AFQ_PREC_MIXED, walkers=walkers)
    e.calculate_mixed_density_matrix()
    e.get_vbias()
    out = {"Gc": e.copy_out("Gc"), "vbias": e.copy_out("vbias")}
    e.sigma(3, 1)
    e.get_vHS()
    out["vHS"] = e.copy_out("vHS")
    e.propagate()
    out["W"] = e.get_walkers()[0]
    e.calculate_mixed_density_matrix()
    out["E"] = e.calculate_energy("chol")
    out["parts"] = e.copy_out("energy_parts")
    out["tuning"] = e.tuning()
    e.close()
    return out


def walkers(s, nw, seed=0, amp=0.05):
    rng = np.random.default_rng(seed)
    W, Wd = s.initial_walkers(nw)
    W = W + amp * (rng.normal(size=W.shape) + 1j * rng.normal(size=W.shape))
    Wd[:, 1] = rng.uniform(0.5, 1.5, nw)
    return W, Wd


@pytest.mark.parametrize("name,kw,nw", [("C1", {}, 16), ("C2", dict(with_vakbl=False), 64)])
def test_forced_kernels_agree(name, kw, nw, monkeypatch):
    s = system(name, **kw)
    wk = walkers(s, nw)
    res = {}
    for force in ("1", "2"):
        monkeypatch.setenv("AFQ_TUNE", force)
        res[force] = run_step(s, nw, wk)
    a, b = res["1"], res["2"]
    for site in ("vhs", "propagate", "t1"):
        assert a["tuning"][site]["kernel"] == 1 and b["tuning"][site]["kernel"] == 2
        assert a["tuning"][site]["ms"][0] > 0 and b["tuning"][site]["ms"][1] > 0
    # the split-K products promote their accumulator: persistent kernel only (forcing the
    # per-tile kernel leaves the built-in rule)
    assert a["tuning"]["splitk"]["kernel"] == 1 and b["tuning"]["splitk"]["kernel"] == 0
    # the per-tile exchange exists for every width, the staged persistent one for 2n in
    # {32, 64, 96} only (C1: 2n = 32, C2: 2n = 64); other widths keep the built-in rule
    assert b["tuning"]["exchange_subset"]["kernel"] == 2
    assert a["tuning"]["exchange_subset"]["kernel"] == (1 if 2 * s.n in (32, 64, 96) else 0)
    for k in ("Gc", "vbias", "vHS", "W"):
        assert rel(a[k], b[k]) < 1e-12, k
    assert rel(a["parts"][:, :2], b["parts"][:, :2]) < 1e-12
    # E_K: promoted persistent exchange against the per-tile one (its accumulator chains
    # over the whole K, so it carries the truncation bias, ~4e-6 relative at C4)
    assert rel(a["parts"][:, 2], b["parts"][:, 2]) < 1e-5
    assert abs(a["E"] - b["E"]) < 1e-5 * abs(b["E"])


def test_timed_choice_cached_per_shape(tmp_path, monkeypatch):
    """The timed choice is one of the candidates, matches a forced run's results, is
    reused by a second handle of the same shape and is written to AFQ_TUNE_CACHE."""
    path = tmp_path / "tune.txt"
    monkeypatch.delenv("AFQ_TUNE", raising=False)
    monkeypatch.setenv("AFQ_TUNE_CACHE", str(path))
    s = system("C2", with_vakbl=False)
    nw = 32
    wk = walkers(s, nw, seed=1)
    t1 = run_step(s, nw, wk)
    t2 = run_step(s, nw, wk)
    tun = t1["tuning"]
    for site in ("vhs", "propagate", "splitk", "exchange_all", "exchange_subset", "t1"):
        assert tun[site]["kernel"] in (1, 2)
        k = tun[site]["kernel"]
        assert tun[site]["ms"][k - 1] > 0
    assert tun["splitk_slices"] >= 1
    assert t2["tuning"] == tun
    for k in ("Gc", "vbias", "vHS", "W", "parts"):
        assert np.array_equal(t1[k], t2[k]), k
    lines = [ln.split() for ln in path.read_text().splitlines() if ln.strip()]
    assert len(lines) == 1 and lines[0][0].startswith("N128_n32_nc512_nw32_")
    assert int(lines[0][-2]) == tun["splitk_slices"]
    assert int(lines[0][-1]) == tun["propagate_walker_group"]["walkers"]
    assert [int(lines[0][1 + 3 * i]) for i in range(6)] == [
        tun[s_]["kernel"] for s_ in ("vhs", "propagate", "splitk", "exchange_all",
                                     "exchange_subset", "t1")]
    # the density matrix precedes the split-K products: equal to a forced run's
    monkeypatch.setenv("AFQ_TUNE", "1" if tun["t1"]["kernel"] == 1 else "2")
    f = run_step(s, nw, wk)
    assert rel(t1["Gc"], f["Gc"]) < 1e-12


@pytest.mark.parametrize("kw", [{}, dict(density=0.3, nchol=128)])
def test_fp64_shapes_do_not_change_results(kw, monkeypatch):
    """FP64 form: the tuner's CTA / tile shapes (CSR vHS, ZGEMM propagation, dense vbias,
    Coulomb and Vakbl) sum every output in the same order, so a tuned handle and one on
    the built-in rules (AFQ_TUNE=0) give bit-identical walkers and energies when both
    multiply each sparse operand the same way (dense tile or CSR); when the tuner measured
    the other product faster for some operand, only the summation order differs (1e-12)."""
    from miniafqmc_b200.afqmc import AfqmcSys, AFQ_PREC_FP64
    s = system("C1", **kw)
    nw = 16
    wk = walkers(s, nw, seed=2)
    out = {}
    for tune in ("0", None):
        if tune is None:
            monkeypatch.delenv("AFQ_TUNE", raising=False)
        else:
            monkeypatch.setenv("AFQ_TUNE", tune)
        e = AfqmcSys(s, nw, precision=AFQ_PREC_FP64, walkers=wk)
        e.calculate_mixed_density_matrix()
        for st in range(6):
            e.substep(4, st, 5, graph=True)
        e.calculate_mixed_density_matrix()
        out[tune] = (e.get_walkers(), e.calculate_energy("chol"), e.calculate_energy("vakbl"),
                     e.tuning(), e.sparse_paths())
        e.close()
    (W0, D0), ec0, ev0, t0, p0 = out["0"]
    (W1, D1), ec1, ev1, t1, p1 = out[None]
    assert all(v["shape"] == 0 for v in t0.values())
    assert t1["vhs_csr"]["ms"][0] > 0 and t1["propagate_zgemm"]["ms"][0] > 0
    if kw:   # dense SpvnT above the density threshold
        assert t1["vbias_zgemm"]["ms"][0] > 0
    # the rule: dense at 25% density and above
    assert p0["Spvn"]["path"] == ("dense" if kw else "csr")
    # the tuner timed both products of every operand dense enough for a dense copy
    assert p1["SpvnT"]["ms"][0] > 0 and p1["SpvnT"]["ms"][1] > 0
    if [v["path"] for v in p0.values()] == [v["path"] for v in p1.values()]:
        assert np.array_equal(W0, W1) and np.array_equal(D0, D1)
        assert ec0 == ec1 and ev0 == ev1
    else:
        assert rel(W1, W0) < 1e-12 and rel(D1, D0) < 1e-12
        assert abs(ec1 - ec0) < 1e-12 * abs(ec0) and abs(ev1 - ev0) < 1e-12 * abs(ev0)


def test_grouped_propagation_chain_is_bit_identical(monkeypatch):
    """The mixed propagation chain run walker group by walker group (AFQ_PROP_GROUP) gives
    the walkers of the chain over all walkers at once, bit for bit (same tiles, same
    epilogues, another launch order), through graph substeps with a re-orthogonalisation.
    The kernel of every product site and the split-K slice count are forced (AFQ_TUNE=1,
    AFQ_SPLITK) so the two handles' separate tuning runs cannot pick different ones (other
    kernel choices agree to 1e-12, not bit for bit)."""
    from miniafqmc_b200.afqmc import AfqmcSys, AFQ_PREC_MIXED
    monkeypatch.setenv("AFQ_TUNE", "1")
    monkeypatch.setenv("AFQ_SPLITK", "2")
    s = system("C2", with_vakbl=False)
    nw = 80
    wk = walkers(s, nw, seed=6)
    out = {}
    for grp in ("0", "32"):
        monkeypatch.setenv("AFQ_PROP_GROUP", grp)
        e = AfqmcSys(s, nw, precision=AFQ_PREC_MIXED, walkers=wk, use_vakbl=False)
        assert e.tuning()["propagate_walker_group"]["walkers"] == int(grp)
        e.calculate_mixed_density_matrix()
        for st in range(6):
            e.substep(9, st, 5, graph=True)
        out[grp] = e.get_walkers()
        e.close()
    assert np.array_equal(out["0"][0], out["32"][0])
    assert np.array_equal(out["0"][1], out["32"][1])


def test_staged_propagation_epilogue_matches_tile_epilogue(monkeypatch):
    """Walker width 2n = 24 (C5's smallest system, not a multiple of 32): the propagation
    products with the staged epilogue on the persistent kernel (AFQ_TUNE=1; Im columns
    gathered from 32-column-aligned TMEM loads) and with the shared-memory tile epilogue on
    the per-tile kernel (AFQ_TUNE=2) do the same arithmetic: walkers to 1e-12 as for the
    other forced-kernel pairs."""
    import dataclasses
    from miniafqmc_b200.synthetic import C5_SYSTEMS, make_system
    cfg = dataclasses.replace(C5_SYSTEMS[0], nwalk=24)
    s = make_system(cfg)
    wk = walkers(s, cfg.nwalk, seed=7)
    res = {}
    for force in ("1", "2"):
        monkeypatch.setenv("AFQ_TUNE", force)
        res[force] = run_step(s, cfg.nwalk, wk)
    a, b = res["1"], res["2"]
    assert a["tuning"]["propagate"]["kernel"] == 1 and b["tuning"]["propagate"]["kernel"] == 2
    assert rel(a["W"], b["W"]) < 1e-12


@pytest.mark.parametrize("wave", ["24", "16"])
def test_fused_propagation_chain_matches_eight_launches(wave, monkeypatch):
    """The propagation chain as one cooperative persistent launch (walker waves, per-walker
    dependency counters, plain products two K slabs per stage) runs the same tiles, MMA
    order and epilogue arithmetic as the eight launches: walkers bit for bit through graph
    substeps with a re-orthogonalisation.  80 walkers in waves of 24 (two full pairs'
    worth of waves and a partial wave of 8) or 16 (five full waves)."""
    from miniafqmc_b200.afqmc import AfqmcSys, AFQ_PREC_MIXED
    monkeypatch.setenv("AFQ_TUNE", "1")
    monkeypatch.setenv("AFQ_SPLITK", "2")
    s = system("C2", with_vakbl=False)
    nw = 80
    wk = walkers(s, nw, seed=8)
    out = {}
    for ch in ("0", wave):
        monkeypatch.setenv("AFQ_PROP_CHAIN", ch)
        e = AfqmcSys(s, nw, precision=AFQ_PREC_MIXED, walkers=wk, use_vakbl=False)
        assert e.tuning()["propagate_chain"]["wave"] == int(ch)
        e.calculate_mixed_density_matrix()
        for st in range(6):
            e.substep(9, st, 5, graph=True)
        out[ch] = e.get_walkers()
        e.close()
    assert np.array_equal(out["0"][0], out[wave][0])
    assert np.array_equal(out["0"][1], out[wave][1])
