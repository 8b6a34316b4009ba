"""The miniapp's driver loop (src/miniapps/miniafqmc_base.cpp:226-349) over an engine.

An engine is anything with the operation interface of `miniafqmc_b200.afqmc.AfqmcSys`
(calculate_mixed_density_matrix, get_vbias, sigma, get_vHS, propagate,
calculate_overlaps, update_weights[_partial], orthogonalize, calculate_energy /
energy_sums, eshift, substep).  With `comm` set, the walker ensemble is sharded: each
rank holds a contiguous block of walkers, draws the auxiliary fields of its block from
the global Philox stream, and the two ensemble couplings of the reference -- Eshift
(miniafqmc_base.cpp:317-327) and the weighted energy (afqmc_sys.hpp:127-132) -- become
sums all-reduced across ranks.
"""
from __future__ import annotations

import dataclasses
from typing import Callable, Optional


@dataclasses.dataclass
class Comm:
    """Walker sharding: this rank holds walkers [offset, offset + nwalk_local) of
    nwalk_global; allreduce(list[float]) -> list[float] sums across ranks."""
    offset: int
    nwalk_global: int
    allreduce: Callable


@dataclasses.dataclass
class RunResult:
    energies: list
    steps: int
    substeps: int


def energy(engine, mode: str = "auto", comm: Optional[Comm] = None) -> float:
    """Eav = sum Re(eloc) Re(w) / sum Re(w) over the whole ensemble."""
    if comm is None:
        return engine.calculate_energy(mode)
    s = engine.energy_sums(mode)
    tot = comm.allreduce([float(s[0]), float(s[1])])
    return tot[0] / tot[1]


def substep(engine, seed: int, step_tot: int, northo: int, comm: Optional[Comm] = None,
            graph: bool = True):
    if comm is None:
        engine.substep(seed, step_tot, northo, graph=graph)
        return
    engine.calculate_mixed_density_matrix()
    engine.get_vbias()
    engine.sigma(seed, step_tot)
    engine.get_vHS()
    engine.propagate()
    engine.calculate_overlaps(save_old=True)
    local = engine.update_weights_partial()
    tot = comm.allreduce([local])[0]
    engine.eshift = tot / comm.nwalk_global          # miniafqmc_base.cpp:327
    if step_tot > 0 and step_tot % northo == 0:     # miniafqmc_base.cpp:330-337
        engine.orthogonalize()
        engine.calculate_overlaps(save_old=False)


def run(engine, nsteps: int, nsubsteps: int, northo: int, seed: int,
        energy_mode: str = "auto", comm: Optional[Comm] = None, graph: bool = True,
        on_energy: Optional[Callable] = None) -> RunResult:
    """nsteps outer steps of nsubsteps propagation substeps, energy after each outer
    step (miniafqmc_base.cpp:249-349); the initial DM + energy (:239-240) included."""
    if comm is not None:
        engine.set_walker_offset(comm.offset, comm.nwalk_global)
    engine.calculate_mixed_density_matrix()
    energies = [energy(engine, energy_mode, comm)]
    step_tot = 0
    for step in range(nsteps):
        for _ in range(nsubsteps):
            substep(engine, seed, step_tot, northo, comm, graph)
            step_tot += 1
        engine.calculate_mixed_density_matrix()
        e = energy(engine, energy_mode, comm)
        energies.append(e)
        if on_energy is not None:
            on_energy(step, e)
    return RunResult(energies, nsteps, step_tot)
