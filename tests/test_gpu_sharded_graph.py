"""Walker-sharded substeps with the Eshift coupling on the device: afq_substep_begin (CUDA
graph up to the weight update, this block's sum of Re W_data[:,4] in a device double),
an NCCL all-reduce of that double on the handle's stream, afq_substep_end (Eshift = sum /
walkers of the ensemble, re-orthogonalisation when scheduled).  With one rank (one GPU
here) every substep must equal afq_substep bit for bit, in both numerical forms; the
reference's coupling is miniafqmc_base.cpp:317-327."""
import numpy as np
import pytest

from conftest import system

pytestmark = pytest.mark.gpu


@pytest.fixture
def nccl_one_rank(tmp_path):
    import torch.distributed as dist
    store = dist.FileStore(str(tmp_path / "store"), 1)
    dist.init_process_group("nccl", store=store, rank=0, world_size=1)
    yield dist
    dist.destroy_process_group()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_device_coupled_substeps_equal_plain(prec, nccl_one_rank):
    import torch
    from miniafqmc_b200 import driver
    from miniafqmc_b200.afqmc import AfqmcSys, AFQ_PREC_FP64, AFQ_PREC_MIXED
    dist = nccl_one_rank
    p = AFQ_PREC_FP64 if prec == "fp64" else AFQ_PREC_MIXED
    s = system("C1")
    nw = 16
    a = AfqmcSys(s, nw, precision=p)
    b = AfqmcSys(s, nw, precision=p)
    calls = []

    def host_allreduce(vals):
        calls.append(vals)
        return vals

    comm = driver.Comm(0, nw, host_allreduce, driver.nccl_allreduce_device(torch, dist))
    b.set_walker_offset(0, nw)
    for e in (a, b):
        e.calculate_mixed_density_matrix()
    for st in range(8):                    # step_tot 3 and 6 re-orthogonalise
        a.substep(4, st, 3, graph=True)
        driver.substep(b, 4, st, 3, comm, graph=True)
    assert not calls                       # the coupling never went through the host
    Wa, Da = a.get_walkers()
    Wb, Db = b.get_walkers()
    assert np.array_equal(Wa, Wb) and np.array_equal(Da, Db)
    assert a.eshift == b.eshift
    a.close()
    b.close()


def test_substep_end_needs_its_begin():
    from miniafqmc_b200.afqmc import AfqmcSys, AfqmcError
    e = AfqmcSys(system("C1"), 16)
    with pytest.raises(AfqmcError):
        e.substep_end(0, 5)
    e.substep_begin(1, 0)
    with pytest.raises(AfqmcError):
        e.substep_end(3, 5)                # not the step that began
    e.substep_end(0, 5)
    e.close()
