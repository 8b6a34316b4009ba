"""Walker sharding across ranks (gloo, world size 2, CPU): the sharded driver with the
oracle as engine reproduces the unsharded ensemble -- same auxiliary fields (global
Philox indexing), same Eshift (all-reduced sum of Re W_data[:,4]) and same weighted
energy (all-reduced sums); per-rank checkpoints resume the sharded run exactly.
Population control is per block: each rank combs its own walkers with the uniform of its
walker offset (independent combs), and no weight moves between ranks."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

NW, STEPS, SUB, NORTHO, SEED = 6, 2, 3, 2, 17


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        from conftest import tiny_system
        from oracle import oracle as O
        from miniafqmc_b200 import driver
        s = tiny_system()
        per = NW // world
        eng = O.Oracle(s, per)

        def allreduce(vals):
            t = torch.tensor(vals, dtype=torch.float64)
            dist.all_reduce(t)
            return t.tolist()

        comm = driver.Comm(rank * per, NW, allreduce)
        res = driver.run(eng, STEPS, SUB, NORTHO, SEED, comm=comm, graph=False)
        W, Wd = eng.get_walkers()
        # the same run with a per-rank checkpoint after the first step, resumed by a new
        # engine on every rank
        ck = os.path.join(out_dir, f"ck{rank}.bin")
        driver.run(O.Oracle(s, per), 1, SUB, NORTHO, SEED, comm=comm, graph=False,
                   checkpoint=ck)
        res2 = driver.run(O.Oracle(s, per), STEPS, SUB, NORTHO, 0, comm=comm, graph=False,
                          resume=driver.read_checkpoint(ck))
        # one comb of this rank's block after the run
        Wb, Wdb = eng.get_walkers()
        eng.population_control(SEED, 99)
        Wc, Wdc = eng.get_walkers()
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), W=W, Wd=Wd, E=np.array(res.energies),
                 E_resumed=np.array(res2.energies), Wb=Wb, Wdb=Wdb, Wc=Wc, Wdc=Wdc)
    finally:
        dist.destroy_process_group()


def test_sharded_run_matches_single_ensemble(tmp_path):
    from conftest import tiny_system
    from oracle import oracle as O
    from miniafqmc_b200 import driver
    s = tiny_system()
    ref = O.Oracle(s, NW)
    res = driver.run(ref, STEPS, SUB, NORTHO, SEED, graph=False)
    Wr, Wdr = ref.get_walkers()
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    parts = [np.load(tmp_path / f"r{r}.npz") for r in range(world)]
    W = np.concatenate([p["W"] for p in parts])
    Wd = np.concatenate([p["Wd"] for p in parts])
    np.testing.assert_allclose(W, Wr, rtol=0, atol=1e-12 * np.abs(Wr).max())
    np.testing.assert_allclose(Wd, Wdr, rtol=1e-11, atol=1e-12)
    for p in parts:
        np.testing.assert_allclose(p["E"], res.energies, rtol=1e-12)
        # per-rank checkpoints resume the sharded run: the steps after it repeat it
        assert np.array_equal(p["E_resumed"][1:], p["E"][2:])
    # sharded population control: block r combs alone with the uniform of offset r * per
    per = NW // world
    for r, p in enumerate(parts):
        We, Wde, _ = O.comb(p["Wb"], p["Wdb"], SEED, 99, offset=r * per)
        assert np.array_equal(p["Wc"], We) and np.array_equal(p["Wdc"], Wde)
        tot = np.maximum(p["Wdb"][:, 1].real, 0).sum()
        assert abs(p["Wdc"][:, 1].real.sum() - tot) < 1e-12 * per * max(tot, 1.0)
    assert O.comb_uniform(SEED, 99, 0) != O.comb_uniform(SEED, 99, per)


class _DeviceCoupledEngine:
    """Stand-in engine with the split substep of a device-coupled sharded run: begin
    leaves this block's e4 sum at an address, end sets Eshift from the summed value."""

    def __init__(self, e4, nwg):
        self.slots = {7: float(e4)}
        self.nwg, self.eshift, self.stream = nwg, None, 0

    def substep_begin(self, seed, step):
        return 7

    def substep_end(self, step, northo):
        self.eshift = self.slots[7] / self.nwg


def _coupled_worker(rank, world, port, out_dir):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        from miniafqmc_b200 import driver
        eng = _DeviceCoupledEngine(10.0 * (rank + 1), 8)

        def allreduce_device(addr, stream):   # gloo stand-in for the NCCL all-reduce
            t = torch.tensor([eng.slots[addr]], dtype=torch.float64)
            dist.all_reduce(t)
            eng.slots[addr] = float(t.item())

        def host(vals):
            raise AssertionError("host all-reduce used")

        comm = driver.Comm(rank * 4, 8, host, allreduce_device)
        driver.substep(eng, 1, 0, 5, comm, graph=True)
        np.save(os.path.join(out_dir, f"e{rank}.npy"), np.array([eng.eshift]))
    finally:
        dist.destroy_process_group()


def test_device_coupled_substep_driver_logic(tmp_path):
    """driver.substep with Comm.allreduce_device: begin, one in-place all-reduce of the
    block sums, end; every rank ends with Eshift = (sum over ranks) / walkers."""
    world = 2
    mp.start_processes(_coupled_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    for r in range(world):
        assert np.load(tmp_path / f"e{r}.npy")[0] == (10.0 + 20.0) / 8
