"""Parity of the sm_100a FP64 path with the FP64 CPU oracle, through the C ABI.

Tolerance: 1e-10 relative (max |gpu - oracle| / max |oracle| per quantity) for every
stage and over whole trajectories -- the bar for the plain FP64 form."""
import dataclasses

import numpy as np
import pytest

from conftest import system, tiny_system
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-10


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def engines(s, nw, walkers=None, **kw):
    from miniafqmc_b200.afqmc import AfqmcSys
    g = AfqmcSys(s, nw, walkers=walkers, **kw)
    o = O.Oracle(s, nw)
    if walkers is not None:
        o.set_walkers(*walkers)
    return g, o


def perturbed(s, nw, seed=0, amp=0.05):
    rng = np.random.default_rng(seed)
    W, Wd = s.initial_walkers(nw)
    W = W + amp * (rng.normal(size=W.shape) + 1j * rng.normal(size=W.shape))
    Wd[:, 1] = rng.uniform(0.5, 1.5, nw)
    return W, Wd


def check_stages(s, nw, seed=3, step=0):
    g, o = engines(s, nw, walkers=perturbed(s, nw))
    for e in (g, o):
        e.calculate_mixed_density_matrix()
    assert rel(g.copy_out("Gc"), o.copy_out("Gc")) < TOL
    assert rel(g.get_walker_data()[:, 2:4], o.get_walkers()[1][:, 2:4]) < TOL
    for e in (g, o):
        e.get_vbias()
    assert rel(g.copy_out("vbias"), o.copy_out("vbias")) < TOL
    for e in (g, o):
        e.sigma(seed, step)
    assert rel(g.copy_out("xraw"), o.copy_out("xraw")) < 1e-13
    assert rel(g.copy_out("X"), o.copy_out("X")) < TOL
    assert rel(g.copy_out("hybridW"), o.copy_out("hybridW")) < TOL
    for e in (g, o):
        e.get_vHS()
    assert rel(g.copy_out("vHS"), o.copy_out("vHS")) < TOL
    for e in (g, o):
        e.propagate()
    assert rel(g.get_walkers()[0], o.get_walkers()[0]) < TOL
    for e in (g, o):
        e.calculate_overlaps(save_old=True)
        e.update_weights()
    assert rel(g.get_walker_data(), o.get_walkers()[1]) < TOL
    assert g.eshift == pytest.approx(o.eshift, rel=TOL)
    for e in (g, o):
        e.orthogonalize()
        e.calculate_overlaps()
    assert rel(g.get_walkers()[0], o.get_walkers()[0]) < TOL
    assert rel(g.get_walker_data(), o.get_walkers()[1]) < TOL
    for e in (g, o):
        e.calculate_mixed_density_matrix()
    modes = (["vakbl"] if s.Vakbl is not None else []) + ["chol"]
    for mode in modes:
        eg, eo = g.calculate_energy(mode), o.calculate_energy(mode)
        assert eg == pytest.approx(eo, rel=TOL), mode
        assert rel(g.get_walker_data()[:, 0], o.get_walkers()[1][:, 0]) < TOL
    g.close()


def test_stages_C1():
    check_stages(system("C1"), 16)


def test_stages_complex_trial_and_cholesky():
    """Complex trial (random unitary rotation) and complex Cholesky vectors exercise every
    conjugation and the complex-valued Spvn path."""
    check_stages(system("C1", complex_trial=True, complex_chol=True, nchol=96, seed=5), 10)


def test_stages_ragged_sizes():
    """Walker count, NMO and electron count that fill no tile exactly."""
    check_stages(tiny_system(nmo=37, nel=5, nchol=29, density=0.25, seed=9), 5)


def test_stages_C2_shapes():
    """C2 shapes (NMO=128, 32+32 electrons, nchol=512) on 40 walkers."""
    s = system("C2", with_vakbl=False)
    check_stages(s, 40)


def test_trajectory_C1_graph_vs_oracle():
    """The C1 workload (16 walkers, 20 steps, ortho every 5, energy every step) through
    the CUDA-graph substep, against the oracle step by step."""
    s = system("C1")
    cfg = s.cfg
    g, o = engines(s, cfg.nwalk)
    for e in (g, o):
        e.calculate_mixed_density_matrix()
    assert g.calculate_energy("vakbl") == pytest.approx(o.calculate_energy("vakbl"), rel=TOL)
    for st in range(cfg.nsteps):
        g.substep(0, st, cfg.northo, graph=True)
        o.substep(0, st, cfg.northo)
        for e in (g, o):
            e.calculate_mixed_density_matrix()
        eg, eo = g.calculate_energy("vakbl"), o.calculate_energy("vakbl")
        assert eg == pytest.approx(eo, rel=TOL), st
        assert g.calculate_energy("chol") == pytest.approx(eo, rel=TOL), st
    Wg, Wdg = g.get_walkers()
    Wo, Wdo = o.get_walkers()
    assert rel(Wg, Wo) < TOL
    assert rel(Wdg, Wdo) < TOL
    assert g.eshift == pytest.approx(o.eshift, rel=TOL)
    g.close()


def test_graph_substep_equals_op_by_op():
    s = system("C1")
    from miniafqmc_b200.afqmc import AfqmcSys
    a = AfqmcSys(s, 16)
    b = AfqmcSys(s, 16)
    for st in range(7):
        a.substep(4, st, 3, graph=True)
        b.substep(4, st, 3, graph=False)
    np.testing.assert_array_equal(a.get_walkers()[0], b.get_walkers()[0])
    np.testing.assert_array_equal(a.get_walker_data(), b.get_walker_data())
    a.close()
    b.close()


def test_sigma_from_host_buffer():
    s = system("C1")
    g, o = engines(s, 16)
    x = np.random.default_rng(2).normal(size=(s.nchol, 16))
    for e in (g, o):
        e.calculate_mixed_density_matrix()
        e.get_vbias()
        e.sigma_from(x)
    assert rel(g.copy_out("X"), o.copy_out("X")) < TOL
    assert rel(g.copy_out("hybridW"), o.copy_out("hybridW")) < TOL
    g.close()


@pytest.mark.parametrize("tune", ["0", "1"])
def test_stages_dense_tile_spvn(tune, monkeypatch):
    """Spvn at 30% density: the built-in rule (AFQ_TUNE=0) multiplies it as a dense tile
    (vHS by ZGEMM over the densified operand), and the set-up tuner picks the faster of
    the dense and CSR products; either way every stage equals the oracle's."""
    from miniafqmc_b200.afqmc import AfqmcSys
    monkeypatch.setenv("AFQ_TUNE", tune)
    s = system("C1", density=0.3, nchol=128)
    e = AfqmcSys(s, 16)
    paths = e.sparse_paths()
    e.close()
    if tune == "0":
        assert paths["Spvn"]["path"] == "dense" and paths["SpvnT"]["path"] == "dense"
    else:
        assert paths["Spvn"]["ms"][0] > 0 and paths["Spvn"]["ms"][1] > 0
    check_stages(s, 16)
