"""Parity of the FP64 form with the oracle on the larger workloads, and of the mixed form
with the FP64 form on the absolute energy bar.

FP64 form against the oracle, 1e-10 relative (max |gpu - oracle| / max |oracle|):
  C2 as run: NMO=128, 32+32 electrons, nchol=512 (5% nonzero), 256 walkers, CUDA-graph
    substeps, orthogonalisation every 5, energy every 2 substeps (20 substeps);
  C3, C4 and the three C5 systems (NMO 96 / 200 / 320, 12+12 / 40+40 / 64+64 electrons,
    128 / 256 / 384 walkers) on a walker subset: each walker's trajectory depends on the
    others only
    through the weights' energy shift (miniafqmc_base.cpp:317-327), so the GPU runs the
    whole ensemble (512 / 1024 walkers) and the oracle 16 of them, placed at their global
    index for the auxiliary fields (set_walker_offset); W, overlaps, the density matrix
    and the local energies of the 16 must agree, and their weights up to one common
    factor per substep (the two ensembles' Eshift differ).  5 substeps, one of them with
    the orthogonalisation.
Mixed form against the FP64 form: every measured energy along a trajectory on the same
auxiliary fields within 1e-4 Ha (absolute), at C3 (64 of its walkers, 20 substeps) and
C4 (all 1024 walkers, 20 substeps), energies every 5 substeps."""
import os

import numpy as np
import pytest

from conftest import system
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-10
DE_HA = 1e-4


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def threads():
    return max(1, os.cpu_count() or 1)


def test_trajectory_C2_graph_vs_oracle():
    from miniafqmc_b200.afqmc import AfqmcSys
    s = system("C2", with_vakbl=False)
    nw, nsub, every, northo = 256, 20, 2, 5
    g = AfqmcSys(s, nw)
    o = O.Oracle(s, nw, threads=threads())
    for e in (g, o):
        e.calculate_mixed_density_matrix()
    assert g.calculate_energy("chol") == pytest.approx(o.calculate_energy("chol"), rel=TOL)
    for st in range(nsub):
        g.substep(1, st, northo, graph=True)
        o.substep(1, st, northo)
        if (st + 1) % every == 0:
            for e in (g, o):
                e.calculate_mixed_density_matrix()
            eg, eo = g.calculate_energy("chol"), o.calculate_energy("chol")
            assert eg == pytest.approx(eo, rel=TOL), st
    Wg, Wdg = g.get_walkers()
    Wo, Wdo = o.get_walkers()
    assert rel(Wg, Wo) < TOL
    assert rel(Wdg, Wdo) < TOL
    assert g.eshift == pytest.approx(o.eshift, rel=TOL)
    g.close()


def c5_system(i):
    from miniafqmc_b200.synthetic import C5_SYSTEMS, make_system
    return make_system(C5_SYSTEMS[i])


@pytest.mark.parametrize("name,off", [("C3", 256), ("C4", 512), ("C5-0", 64), ("C5-1", 128),
                                      ("C5-2", 192)])
def test_walker_subset_vs_oracle(name, off):
    from miniafqmc_b200.afqmc import AfqmcSys
    s = c5_system(int(name[3:])) if name.startswith("C5-") else system(name)
    cfg = s.cfg
    nw, k, seed, northo, nsub = cfg.nwalk, 16, cfg.seed, 5, 6
    g = AfqmcSys(s, nw, use_vakbl=False)
    o = O.Oracle(s, k, threads=threads())
    o.set_walker_offset(off, nw)
    sl = slice(off, off + k)
    for e in (g, o):
        e.calculate_mixed_density_matrix()
    for st in range(nsub):                 # step_tot 5 re-orthogonalises
        g.substep(seed, st, northo, graph=True)
        o.substep(seed, st, northo)
    Wg, Wdg = g.get_walkers()
    Wo, Wdo = o.get_walkers()
    assert rel(Wg[sl], Wo) < TOL
    assert rel(Wdg[sl, 2:8], Wdo[:, 2:8]) < TOL       # overlaps and hybrid energies
    ratio = Wdg[sl, 1].real / Wdo[:, 1].real          # one common factor
    assert np.max(np.abs(ratio / ratio[0] - 1)) < TOL
    for e in (g, o):
        e.calculate_mixed_density_matrix()
    assert rel(g.copy_out("Gc")[:, sl], o.copy_out("Gc")) < TOL
    g.calculate_energy("chol")
    o.calculate_energy("chol")
    assert rel(g.get_walker_data()[sl, 0], o.get_walkers()[1][:, 0]) < TOL
    g.close()


@pytest.mark.parametrize("name,nw", [("C3", 64), ("C4", 1024)])
def test_mixed_energy_within_absolute_bar(name, nw):
    from miniafqmc_b200.afqmc import AfqmcSys, AFQ_PREC_FP64, AFQ_PREC_MIXED
    s = system(name)
    seed = s.cfg.seed
    d = AfqmcSys(s, nw, precision=AFQ_PREC_FP64, use_vakbl=False)
    m = AfqmcSys(s, nw, precision=AFQ_PREC_MIXED, use_vakbl=False)
    dE = []
    for e in (d, m):
        e.calculate_mixed_density_matrix()
    for st in range(20):
        for e in (d, m):
            e.substep(seed, st, 5, graph=True)
        if (st + 1) % 5 == 0:
            for e in (d, m):
                e.calculate_mixed_density_matrix()
            dE.append(abs(m.calculate_energy("chol") - d.calculate_energy("chol")))
    m.synchronize()
    assert max(dE) < DE_HA, dE
    d.close()
    m.close()
