"""Population control by the comb and exact resume from saved walkers (no reference
counterpart: the reference leaves branching out, miniafqmc_base.cpp:347).

The comb is restated in the oracle (`oracle.comb`: prefix sums in walker order, teeth at
(j + u) T / nw, first walker with C_i > t, the same Philox uniform), and the GPU copies
must equal it exactly.  Resume: a run stopped after five substeps, its walkers, walker
data and Eshift saved and loaded into a fresh handle, continues bit for bit like the run
that never stopped (same seed and step counter)."""
import numpy as np
import pytest

from conftest import system
from oracle import oracle as O

pytestmark = pytest.mark.gpu

comb = O.comb


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_comb_matches_numpy(prec):
    from miniafqmc_b200.afqmc import AfqmcSys, AFQ_PREC_FP64, AFQ_PREC_MIXED
    s = system("C1")
    nw = 64
    rng = np.random.default_rng(11)
    W, Wd = s.initial_walkers(nw)
    W = W + 0.05 * (rng.normal(size=W.shape) + 1j * rng.normal(size=W.shape))
    Wd[:, 1] = rng.lognormal(0.0, 0.8, nw)
    Wd[::7, 1] = 0.0                      # killed walkers
    Wd[3, 1] = -0.5                       # a negative weight counts as zero
    Wd[:, 0] = rng.normal(size=nw)        # walker data that must travel with the copies
    e = AfqmcSys(s, nw, precision=AFQ_PREC_FP64 if prec == "fp64" else AFQ_PREC_MIXED,
                 walkers=(W, Wd))
    W0, Wd0 = e.get_walkers()
    for seed, step in ((7, 3), (7, 4)):    # two combs in a row
        e.population_control(seed, step)
        Wexp, Wdexp, idx = comb(W0, Wd0, seed, step)
        W1, Wd1 = e.get_walkers()
        assert np.array_equal(W1, Wexp) and np.array_equal(Wd1, Wdexp)
        assert abs(Wd1[:, 1].real.sum() - np.maximum(Wd0[:, 1].real, 0).sum()) < 1e-12 * nw
        assert not np.any(np.isin(idx, np.nonzero(Wd0[:, 1].real <= 0)[0]))
        W0, Wd0 = W1, Wd1
    e.close()


def test_comb_of_a_sharded_block_uses_its_offset():
    """A handle holding walkers [offset, offset + nw) of a larger ensemble combs its block
    with the uniform of its offset (oracle.comb with offset=)."""
    from miniafqmc_b200.afqmc import AfqmcSys
    s = system("C1")
    nw, off = 32, 32
    rng = np.random.default_rng(12)
    W, Wd = s.initial_walkers(nw)
    Wd[:, 1] = rng.lognormal(0.0, 0.8, nw)
    e = AfqmcSys(s, nw, walkers=(W, Wd))
    e.set_walker_offset(off, 2 * nw)
    W0, Wd0 = e.get_walkers()
    e.population_control(7, 3)
    Wexp, Wdexp, _ = comb(W0, Wd0, 7, 3, offset=off)
    W1, Wd1 = e.get_walkers()
    assert np.array_equal(W1, Wexp) and np.array_equal(Wd1, Wdexp)
    e.close()


def test_comb_rejects_dead_population():
    from miniafqmc_b200.afqmc import AfqmcSys, AfqmcError
    s = system("C1")
    W, Wd = s.initial_walkers(16)
    Wd[:, 1] = 0.0
    e = AfqmcSys(s, 16, walkers=(W, Wd))
    before = e.get_walkers()
    with pytest.raises(AfqmcError):
        e.population_control(1, 1)
    after = e.get_walkers()      # untouched, and the handle still works
    assert np.array_equal(before[0], after[0]) and np.array_equal(before[1], after[1])
    e.close()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_resume_from_saved_walkers_is_exact(prec):
    from miniafqmc_b200.afqmc import AfqmcSys, AFQ_PREC_FP64, AFQ_PREC_MIXED
    p = AFQ_PREC_FP64 if prec == "fp64" else AFQ_PREC_MIXED
    s = system("C1")
    nw, seed, northo = 16, 5, 5

    def run(e, steps):
        for st in steps:
            e.substep(seed, st, northo, graph=True)
            if (st + 1) % 5 == 0:
                e.population_control(seed, st)

    a = AfqmcSys(s, nw, precision=p)
    a.calculate_mixed_density_matrix()
    run(a, range(10))
    Wa, Wda = a.get_walkers()
    ea = a.eshift
    b = AfqmcSys(s, nw, precision=p)
    b.calculate_mixed_density_matrix()
    run(b, range(5))
    saved = b.get_walkers(), b.eshift
    b.close()
    c = AfqmcSys(s, nw, precision=p, walkers=saved[0])
    c.eshift = saved[1]
    c.calculate_mixed_density_matrix()
    run(c, range(5, 10))
    Wc, Wdc = c.get_walkers()
    assert np.array_equal(Wa, Wc) and np.array_equal(Wda, Wdc) and c.eshift == ea
    a.close()
    c.close()
