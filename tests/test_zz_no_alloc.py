"""afq_exchange_energy_noalloc: the exchange energy for callers that cannot allocate
device memory (graph capture, pool-owning frameworks).  Its per-walker output must equal
the exchange part of the handle's Cholesky energy (afq_energy + AFQ_BUF_ENERGY_PARTS) to
1e-10 relative -- the FP64 parity tolerance -- on two calls in a row, since every call
reuses the same static scratch array.  Inputs and outputs are device buffers the test
(the caller) allocates with torch; the entry point itself allocates nothing.  The
argument checks (alignment, batch size) run on the host before any device work, so they
are tested without a GPU."""
import ctypes

import numpy as np
import pytest

from conftest import system

TOL = 1e-10


def _entry():
    from miniafqmc_b200.afqmc import load_library
    lib = load_library()
    f = lib.afq_exchange_energy_noalloc
    f.argtypes = [ctypes.c_void_p] * 2 + [ctypes.c_int] * 4 + [ctypes.c_void_p] * 2
    f.restype = ctypes.c_int
    return f


@pytest.mark.gpu
def test_exchange_energy_noalloc_matches_handle_twice():
    import torch
    from miniafqmc_b200.afqmc import AfqmcSys, load_library
    s = system("C1")
    nw = 16
    rng = np.random.default_rng(4)
    W, Wd = s.initial_walkers(nw)
    W = W + 0.05 * (rng.normal(size=W.shape) + 1j * rng.normal(size=W.shape))
    g = AfqmcSys(s, nw, walkers=(W, Wd))
    g.calculate_mixed_density_matrix()
    g.calculate_energy("chol")
    ek_ref = g.copy_out("energy_parts")[:, 2]
    gc = g.copy_out("Gc")                      # reference layout [2nN][nw]
    g.close()
    lib = load_library()
    lib.afq_exchange_energy_noalloc.argtypes = [ctypes.c_void_p] * 2 + [ctypes.c_int] * 4 + \
        [ctypes.c_void_p] * 2
    lib.afq_exchange_energy_noalloc.restype = ctypes.c_int
    dev = torch.device("cuda", 0)
    lh = torch.from_numpy(np.ascontiguousarray(s.Lh).view(np.float64)).to(dev)
    gcw = torch.from_numpy(np.ascontiguousarray(gc.T).view(np.float64)).to(dev)
    ek = torch.zeros(2 * nw, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        ek.fill_(float("nan"))
        st = lib.afq_exchange_energy_noalloc(lh.data_ptr(), gcw.data_ptr(), s.N, s.n, s.nchol, nw,
                                             ek.data_ptr(), stream)
        torch.cuda.synchronize(dev)
        assert st == 0, (call, st)
        out = ek.cpu().numpy().view(np.complex128)
        err = np.max(np.abs(out.real - ek_ref)) / np.max(np.abs(ek_ref))
        assert err < TOL, (call, err)


def test_exchange_energy_noalloc_rejects_oversized_batch():
    f = _entry()
    # 2 * 4096 walkers * 1536/2 blocks far exceeds the 2^18 partials of the static array
    dummy = ctypes.c_void_p(16)
    assert f(dummy, dummy, 384, 48, 1536, 4096, dummy, None) == 5   # AFQ_ERR_UNSUPPORTED
    # few partials but more than 65535 walker groups in the launch grid (naea > 48: one
    # walker per group)
    assert f(dummy, dummy, 96, 64, 1, 70000, dummy, None) == 5


def test_exchange_energy_noalloc_rejects_misaligned_buffers():
    """The kernels move 16-byte complex values: 8-byte aligned pointers are refused
    before any device work (AFQ_ERR_ARG) instead of faulting on the GPU."""
    f = _entry()
    ok, odd = ctypes.c_void_p(4096), ctypes.c_void_p(4096 + 8)
    for args in ((odd, ok, ok), (ok, odd, ok), (ok, ok, odd)):
        assert f(args[0], args[1], 64, 16, 256, 16, args[2], None) == 1   # AFQ_ERR_ARG
