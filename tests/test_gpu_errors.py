"""Failure paths of the C ABI: bad arguments, calls out of order, and a walker whose
overlap matrix is exactly singular (a zero column planted in its Slater matrix), which the
batched LU reports per walker instead of trapping -- all produced on the host -- and the
tensor-core kernels' bounded pipeline waits, made to run out on an ordinary launch by a
bound of a few hundred clocks (no fault, no hang: every wait ends, the kernel drains its
own copies and MMAs with the default bound before it frees its tensor memory)."""
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


WAIT_CLOCKS = 300   # far below one TMA fill (~1 us): every work wait runs out


def _bf16(x):
    """Rounds float32 values to the nearest bf16 (kept as float32)."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.view(np.float32)


@pytest.mark.parametrize("mode", [0, 1])
def test_tensor_core_wait_timeout_reported_then_recovers(mode):
    """Per-tile (mode 0) and persistent (mode 1) tcgen05 GEMM: with the work-wait bound
    lowered the launch ends with timeout flags and a clean CUDA status; with the default
    bound restored the same launch is correct (fp32 reference of bf16 inputs)."""
    from miniafqmc_b200.afqmc import load_library
    lib = load_library()
    rng = np.random.default_rng(5)
    M, N, K = 256, 128, 2048
    A, B = _bf16(rng.normal(size=(M, K))), _bf16(rng.normal(size=(N, K)))
    C = np.zeros((M, N), np.float32)
    err = ctypes.c_int(0)

    def run():
        return lib.afq_selftest_tc_gemm(M, N, K, 1, 0, 128, mode, A.ctypes.data, B.ctypes.data,
                                        C.ctypes.data, ctypes.byref(err))

    assert lib.afq_set_tc_wait_limit(0, WAIT_CLOCKS) == 0
    try:
        st = run()
    finally:
        assert lib.afq_set_tc_wait_limit(0, 0) == 0
    assert st == 0 and err.value != 0, (st, err.value)
    st = run()
    assert st == 0 and err.value == 0
    ref = A.astype(np.float64) @ B.astype(np.float64).T
    assert np.max(np.abs(C - ref)) < 1e-4 * np.max(np.abs(ref))


def test_handle_reports_timeout_and_next_call_succeeds():
    """Mixed form: a vbias product whose waits run out makes afq_synchronize return the
    timeout status; the flags are cleared once reported, and the same call with the
    default bound gives the vbias of a handle that never timed out."""
    from miniafqmc_b200.afqmc import AfqmcSys, AfqmcError, AFQ_PREC_MIXED, load_library
    lib = load_library()
    s = system("C1")
    ref = AfqmcSys(s, 16, precision=AFQ_PREC_MIXED)
    ref.calculate_mixed_density_matrix()
    ref.get_vbias()
    want = ref.copy_out("vbias")
    ref.close()
    m = AfqmcSys(s, 16, precision=AFQ_PREC_MIXED)
    m.calculate_mixed_density_matrix()
    m.synchronize()
    assert lib.afq_set_tc_wait_limit(0, WAIT_CLOCKS) == 0
    try:
        m.get_vbias()
        with pytest.raises(AfqmcError) as ei:
            m.synchronize()
    finally:
        assert lib.afq_set_tc_wait_limit(0, 0) == 0
    assert ei.value.status == 3 and "timed out" in str(ei.value)
    m.synchronize()                       # reported once, then cleared
    m.get_vbias()
    m.synchronize()
    assert np.array_equal(m.copy_out("vbias"), want)
    m.close()
