"""Failure paths of the C ABI, all produced on the host: bad arguments, calls out of
order, and a walker whose overlap matrix is exactly singular (a zero column planted in
its Slater matrix), which the batched LU reports per walker instead of trapping."""
import ctypes

import numpy as np
import pytest

from conftest import system, tiny_system

pytestmark = pytest.mark.gpu


def test_bad_arguments_and_order():
    from miniafqmc_b200.afqmc import load_library, SystemDesc
    lib = load_library()
    h = ctypes.c_void_p()
    bad = SystemDesc(16, 4, 5, 8, 4, 0.01, 6, 0, 0)   # naea != naeb
    assert lib.afq_create(ctypes.byref(bad), ctypes.byref(h)) == 5
    bad = SystemDesc(16, 4, 4, 8, 0, 0.01, 6, 0, 0)   # no walkers
    assert lib.afq_create(ctypes.byref(bad), ctypes.byref(h)) == 1
    good = SystemDesc(16, 4, 4, 8, 4, 0.01, 6, 0, 0)
    assert lib.afq_create(ctypes.byref(good), ctypes.byref(h)) == 0
    assert lib.afq_vbias(h) == 2                      # no Hamiltonian yet
    assert b"Hamiltonian" in lib.afq_last_error(h)
    assert lib.afq_set_hamiltonian(h, None, None, None, None, None, None, None) == 1
    lib.afq_destroy(h)


def test_singular_walker_is_flagged_not_fatal():
    from miniafqmc_b200.afqmc import AfqmcSys
    s = tiny_system(nmo=16, nel=4, nchol=12, seed=2)
    W, Wd = s.initial_walkers(3)
    W[1, 0, :, 2] = 0.0          # walker 1, spin up: a zero column -> det(T1) = 0
    g = AfqmcSys(s, 3, walkers=(W, Wd))
    g.calculate_mixed_density_matrix()
    info = g.copy_out("info")
    assert info[1, 0] == 1 and info.sum() == 1
    Wd2 = g.get_walker_data()
    assert Wd2[1, 2] == 0
    assert np.all(np.isfinite(g.copy_out("Gc")))
    assert abs(Wd2[0, 2] - 1.0) < 1e-12
    g.close()


def test_walker_offset_validation():
    from miniafqmc_b200.afqmc import AfqmcSys, AfqmcError
    g = AfqmcSys(system("C1"), 16)
    with pytest.raises(AfqmcError):
        g.set_walker_offset(8, 20)      # 8 + 16 > 20
    g.set_walker_offset(16, 32)
    g.close()
