"""Heterogeneous multi-system batch (no reference counterpart): three systems of uneven
NMO, electron count and nchol (the C5 shapes, fewer walkers) advanced by AfqmcBatch with
one graph launch per substep give the same walkers, weights and energies as the same
systems advanced one by one with afq_substep (the same kernels in the same order per
system: equal to 1e-13 relative)."""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

_SYS = {}


def systems():
    if not _SYS:
        from miniafqmc_b200.synthetic import C5_SYSTEMS, make_system
        for i, c in enumerate(C5_SYSTEMS):
            cfg = dataclasses.replace(c, nwalk=(16, 32, 24)[i])
            _SYS[i] = (cfg, make_system(cfg))
    return [_SYS[i] for i in range(len(_SYS))]


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("mixed,nsub", [(False, 1), (True, 1), (True, 5)])
def test_batch_matches_systems_alone(mixed, nsub):
    """nsub substeps per graph launch (nsub = 5: the launches cover substeps 0-4 and 5-9,
    the second one re-orthogonalising in its first substep)."""
    from miniafqmc_b200.afqmc import AfqmcSys, AfqmcBatch, AFQ_PREC_FP64, AFQ_PREC_MIXED
    prec = AFQ_PREC_MIXED if mixed else AFQ_PREC_FP64
    sys_ = systems()
    alone = [AfqmcSys(s, c.nwalk, precision=prec, use_vakbl=False) for c, s in sys_]
    grouped = [AfqmcSys(s, c.nwalk, precision=prec, use_vakbl=False) for c, s in sys_]
    seeds = [c.seed for c, _ in sys_]
    batch = AfqmcBatch(grouped)
    for e in alone + grouped:
        e.calculate_mixed_density_matrix()
    nst = 7 if nsub == 1 else 10   # includes the orthogonalisation at step 5
    for st in range(nst):
        for e, sd in zip(alone, seeds):
            e.substep(sd, st, 5, graph=True)
        if nsub == 1:
            batch.substep(seeds, st, 5)
        elif st % nsub == 0:
            batch.substeps(seeds, st, nsub, 5)
    batch.synchronize()
    for a, g in zip(alone, grouped):
        Wa, Da = a.get_walkers()
        Wg, Dg = g.get_walkers()
        assert rel(Wg, Wa) < 1e-13 and rel(Dg, Da) < 1e-13
        for e in (a, g):
            e.calculate_mixed_density_matrix()
        ea, eg = a.calculate_energy("chol"), g.calculate_energy("chol")
        assert abs(eg - ea) <= 1e-13 * abs(ea)
        assert np.all(np.isfinite(Dg[:, 1].real)) and np.all(Dg[:, 1].real >= 0)
    batch.close()
    for e in alone + grouped:
        e.close()


@pytest.mark.parametrize("mode,nsub", [(3, 1), (3, 5), (1, 5), (2, 5)])
def test_fused_batch_matches_systems_alone(mode, nsub, monkeypatch):
    """Fused batch: the vHS product and each of the eight propagation products run as one
    launch over the three systems' (walker, M tile, N tile) work list.  Every tile runs the
    same MMA sequence and the same epilogue arithmetic as in a system's own launches (the
    system with 2n = 128 takes the tile epilogue and the pack kernels instead of the paired
    epilogue, which writes the same values), so the walkers, weights and energies equal
    the systems advanced alone to 1e-13 relative, through a re-orthogonalisation.  Modes:
    3 both joint, 1 the vHS product only, 2 the chain only.  The joint vHS launch streams
    128-byte K slabs; the set-up tuner may give a system alone the 64-byte-slab epilogue,
    which adds the hi*lo and lo*hi products of every 32 K columns in another order, so the
    systems alone are pinned to a 128-byte-slab epilogue here."""
    from miniafqmc_b200.afqmc import AfqmcSys, AfqmcBatch, AFQ_PREC_MIXED
    monkeypatch.setenv("AFQ_VHS_EPI", "0")
    sys_ = systems()
    alone = [AfqmcSys(s, c.nwalk, precision=AFQ_PREC_MIXED, use_vakbl=False) for c, s in sys_]
    grouped = [AfqmcSys(s, c.nwalk, precision=AFQ_PREC_MIXED, use_vakbl=False) for c, s in sys_]
    seeds = [c.seed for c, _ in sys_]
    batch = AfqmcBatch(grouped)
    batch.set_fused(mode)
    for e in alone + grouped:
        e.calculate_mixed_density_matrix()
    for st in range(10):
        for e, sd in zip(alone, seeds):
            e.substep(sd, st, 5, graph=True)
        if nsub == 1:
            batch.substep(seeds, st, 5)
        elif st % nsub == 0:
            batch.substeps(seeds, st, nsub, 5)
    batch.synchronize()
    for a, g in zip(alone, grouped):
        Wa, Da = a.get_walkers()
        Wg, Dg = g.get_walkers()
        assert rel(Wg, Wa) < 1e-13 and rel(Dg, Da) < 1e-13
        for e in (a, g):
            e.calculate_mixed_density_matrix()
        ea, eg = a.calculate_energy("chol"), g.calculate_energy("chol")
        assert abs(eg - ea) <= 1e-13 * abs(ea)
    # back to the per-system branches: the next substeps still agree
    batch.set_fused(False)
    for e, sd in zip(alone, seeds):
        e.substep(sd, 10, 5, graph=True)
    batch.substep(seeds, 10, 5)
    batch.synchronize()
    for a, g in zip(alone, grouped):
        assert rel(g.get_walkers()[0], a.get_walkers()[0]) < 1e-13
    batch.close()
    for e in alone + grouped:
        e.close()


def test_fused_batch_needs_mixed_systems():
    from miniafqmc_b200.afqmc import AfqmcSys, AfqmcBatch, AfqmcError, AFQ_PREC_FP64, AFQ_PREC_MIXED
    (c0, s0), (c1, s1) = systems()[:2]
    hs = [AfqmcSys(s0, c0.nwalk, precision=AFQ_PREC_MIXED, use_vakbl=False),
          AfqmcSys(s1, c1.nwalk, precision=AFQ_PREC_FP64, use_vakbl=False)]
    batch = AfqmcBatch(hs)
    with pytest.raises(AfqmcError):
        batch.set_fused(True)
    batch.close()
    for e in hs:
        e.close()


def test_c5_shapes_mixed_energy_matches_fp64():
    """Mixed against FP64 energies on identical walkers for the C5 shapes (n = 12, 40 and
    64: promoted exchange tiles of 8 walkers of 24 columns, 2 walkers of 80 columns in a
    160-column tile, 2 walkers of 128 columns): 1e-4 relative on every walker's E_J and E_K,
    and the mean local energy within 1e-4 Ha.  Every width runs the promoted exchange (the
    set-up tuner keeps it: exchange kernel 1)."""
    from miniafqmc_b200.afqmc import AfqmcSys, AFQ_PREC_FP64, AFQ_PREC_MIXED
    rng = np.random.default_rng(3)
    for cfg, s in systems():
        nw = cfg.nwalk
        W, Wd = s.initial_walkers(nw)
        W = W + 0.05 * (rng.normal(size=W.shape) + 1j * rng.normal(size=W.shape))
        parts = []
        for prec in (AFQ_PREC_FP64, AFQ_PREC_MIXED):
            e = AfqmcSys(s, nw, precision=prec, walkers=(W, Wd), use_vakbl=False)
            e.calculate_mixed_density_matrix()
            e.calculate_energy("chol")
            parts.append(e.copy_out("energy_parts"))
            if prec == AFQ_PREC_MIXED:
                tun = e.tuning()
                assert tun["exchange_all"]["kernel"] == 1, (cfg.nel, tun["exchange_all"])
            e.close()
        pd, pm = parts
        ej = rel(pm[:, 1], pd[:, 1])
        ek = rel(pm[:, 2], pd[:, 2])
        assert ej < 1e-4 and ek < 1e-4, (cfg.nmo, cfg.nel, ej, ek)
        de = np.mean((pm[:, 0] + pm[:, 1] - pm[:, 2]) - (pd[:, 0] + pd[:, 1] - pd[:, 2]))
        assert abs(de) < 1e-4, (cfg.nmo, cfg.nel, de)
