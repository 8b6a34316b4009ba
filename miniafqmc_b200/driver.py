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

import numpy as np

CHECKPOINT_MAGIC = b"AFQCKP01"


@dataclasses.dataclass
class Comm:
    """Walker sharding: this rank holds walkers [offset, offset + nwalk_local) of
    nwalk_global; allreduce(list[float]) -> list[float] sums across ranks.  Optional
    allreduce_device(address, stream): sums one float64 at a device address in place
    across ranks, ordered on the given CUDA stream (NCCL); with it, graph substeps of an
    engine that has substep_begin / substep_end keep the Eshift coupling on the device."""
    offset: int
    nwalk_global: int
    allreduce: Callable
    allreduce_device: Optional[Callable] = None


@dataclasses.dataclass
class RunResult:
    energies: list
    steps: int
    substeps: int


class _DeviceDouble:
    """One float64 at a device address, seen through the CUDA array interface."""

    def __init__(self, addr: int):
        self.__cuda_array_interface__ = {"shape": (1,), "typestr": "<f8",
                                         "data": (int(addr), False), "version": 3}


def nccl_allreduce_device(torch, dist) -> Callable:
    """Comm.allreduce_device over torch.distributed (NCCL): the double at `addr` becomes a
    tensor view (no copy) and is summed across ranks on the engine's stream."""
    def allreduce_device(addr: int, stream: int):
        t = torch.as_tensor(_DeviceDouble(addr), device="cuda")
        with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
            dist.all_reduce(t)
    return allreduce_device


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
    if graph and comm.allreduce_device is not None and hasattr(engine, "substep_begin"):
        addr = engine.substep_begin(seed, step_tot)
        comm.allreduce_device(addr, engine.stream)
        engine.substep_end(step_tot, northo)
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


def write_checkpoint(path: str, engine, steps: int, step_tot: int, seed: int,
                     precision: int = 0) -> None:
    """Everything a substep reads besides the Hamiltonian, in the driver program's layout
    (`miniafqmc_b200/app/miniafqmc.cpp`, so either driver resumes the other's runs):
    "AFQCKP01"; int32 nmo, naea, nwalk, precision; int64 steps, step_tot; uint64 seed;
    float64 eshift; complex128 W[nwalk][2][nmo][naea]; complex128 W_data[nwalk][8]."""
    W, Wd = engine.get_walkers()
    nwalk, _, nmo, naea = W.shape
    with open(path, "wb") as f:
        f.write(CHECKPOINT_MAGIC)
        f.write(np.array([nmo, naea, nwalk, precision], "<i4").tobytes())
        f.write(np.array([steps, step_tot], "<i8").tobytes())
        f.write(np.array([seed], "<u8").tobytes())
        f.write(np.array([engine.eshift], "<f8").tobytes())
        f.write(np.ascontiguousarray(W, "<c16").tobytes())
        f.write(np.ascontiguousarray(Wd, "<c16").tobytes())


def read_checkpoint(path: str) -> dict:
    buf = open(path, "rb").read()
    if buf[:8] != CHECKPOINT_MAGIC or len(buf) < 48:
        raise ValueError(f"{path}: not a checkpoint file")
    nmo, naea, nwalk, precision = (int(v) for v in np.frombuffer(buf, "<i4", 4, 8))
    steps, step_tot = (int(v) for v in np.frombuffer(buf, "<i8", 2, 24))
    seed = int(np.frombuffer(buf, "<u8", 1, 40)[0])
    eshift = float(np.frombuffer(buf, "<f8", 1, 48)[0])
    nW, nD = nwalk * 2 * nmo * naea, nwalk * 8
    if len(buf) != 56 + 16 * (nW + nD):
        raise ValueError(f"{path}: walker arrays do not match the header")
    W = np.frombuffer(buf, "<c16", nW, 56).reshape(nwalk, 2, nmo, naea).copy()
    Wd = np.frombuffer(buf, "<c16", nD, 56 + 16 * nW).reshape(nwalk, 8).copy()
    return {"nmo": nmo, "naea": naea, "nwalk": nwalk, "precision": precision,
            "steps": steps, "step_tot": step_tot, "seed": seed, "eshift": eshift,
            "W": W, "W_data": Wd}


def run(engine, nsteps: int, nsubsteps: int, northo: int, seed: int,
        energy_mode: str = "auto", comm: Optional[Comm] = None, graph: bool = True,
        on_energy: Optional[Callable] = None, resume: Optional[dict] = None,
        checkpoint: Optional[str] = None, branch_every: int = 0) -> RunResult:
    """nsteps outer steps of nsubsteps propagation substeps, energy after each outer
    step (miniafqmc_base.cpp:249-349); the initial DM + energy (:239-240) included.
    `resume` (a `read_checkpoint` dict) restores the walkers, Eshift, seed and step
    counters and runs the steps from there up to nsteps; `checkpoint` writes one after
    the last step.  With `comm`, every rank checkpoints and resumes its own walker block
    (one file per rank; Eshift is the ensemble's on every rank).  `branch_every` = k > 0
    runs population control (the comb, `population_control(seed, step_tot)`) after every
    k-th step's energy, where the miniapp marks that branching belongs
    (miniafqmc_base.cpp:347); sharded walker sets comb their own block, each with the
    comb uniform of its walker offset, so the blocks resample independently and keep
    their own total weight (this differs from one comb over the whole ensemble)."""
    if comm is not None:
        engine.set_walker_offset(comm.offset, comm.nwalk_global)
    step0 = step_tot = 0
    if resume is not None:
        engine.set_walkers(resume["W"], resume["W_data"])
        engine.eshift = resume["eshift"]
        step0, step_tot, seed = resume["steps"], resume["step_tot"], resume["seed"]
    engine.calculate_mixed_density_matrix()
    energies = [energy(engine, energy_mode, comm)]
    for step in range(step0, nsteps):
        for _ in range(nsubsteps):
            substep(engine, seed, step_tot, northo, comm, graph)
            step_tot += 1
        engine.calculate_mixed_density_matrix()
        e = energy(engine, energy_mode, comm)
        energies.append(e)
        if on_energy is not None:
            on_energy(step, e)
        if branch_every > 0 and (step + 1) % branch_every == 0:
            engine.population_control(seed, step_tot)
    if checkpoint is not None:
        write_checkpoint(checkpoint, engine, max(nsteps, step0), step_tot, seed)
    return RunResult(energies, nsteps, step_tot)
