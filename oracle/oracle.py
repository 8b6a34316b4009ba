"""ctypes wrapper around the FP64 CPU oracle (`oracle/afqmc_oracle.cpp`).

TEST INFRASTRUCTURE ONLY: imported by tests/, `__graft_entry__.smoke()` and the
`cpu_baseline` / `--impl reference` legs of bench.py.  The product never imports it.

BLAS/LAPACK come from scipy's bundled OpenBLAS (scipy 1.18.1 here): the Fortran-ABI
function pointers are read out of `scipy.linalg.cython_blas` / `cython_lapack`
capsules and handed to the oracle, which then calls zgemm/zgemv/zgetrf/zgetri/
zgelqf/zunglq exactly where the reference does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_EXACT = os.path.join(HERE, "liborc.so")        # -O2, IEEE arithmetic (parity)
LIB_FAST = os.path.join(HERE, "liborc_fast.so")    # reference Release flags (timing)
SRC = os.path.join(HERE, "afqmc_oracle.cpp")

# Reference GNU Release flags: CMake/GNUCompilers.cmake:8-9,27-28
FLAGS_EXACT = ["-O2", "-fopenmp", "-std=c++17", "-fPIC", "-shared"]
FLAGS_FAST = ["-O3", "-ffast-math", "-fopenmp", "-std=c++17", "-fPIC", "-shared"]


def build(force: bool = False) -> None:
    for out, flags in ((LIB_EXACT, FLAGS_EXACT), (LIB_FAST, FLAGS_FAST)):
        if force or not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(SRC):
            subprocess.check_call(["g++", *flags, SRC, "-o", out])


def _capsule_ptr(mod, name: str) -> int:
    cap = mod.__pyx_capi__[name]
    ctypes.pythonapi.PyCapsule_GetName.restype = ctypes.c_char_p
    ctypes.pythonapi.PyCapsule_GetName.argtypes = [ctypes.py_object]
    ctypes.pythonapi.PyCapsule_GetPointer.restype = ctypes.c_void_p
    ctypes.pythonapi.PyCapsule_GetPointer.argtypes = [ctypes.py_object, ctypes.c_char_p]
    return ctypes.pythonapi.PyCapsule_GetPointer(cap, ctypes.pythonapi.PyCapsule_GetName(cap))


_LIBS: dict = {}


def load(fast: bool = False) -> ctypes.CDLL:
    path = LIB_FAST if fast else LIB_EXACT
    if path in _LIBS:
        return _LIBS[path]
    if not os.path.exists(path):
        build()
    lib = ctypes.CDLL(path)
    import scipy.linalg.cython_blas as cb
    import scipy.linalg.cython_lapack as cl
    ptrs = [_capsule_ptr(cb, "zgemm"), _capsule_ptr(cb, "zgemv"),
            _capsule_ptr(cl, "zgetrf"), _capsule_ptr(cl, "zgetri"),
            _capsule_ptr(cl, "zgelqf"), _capsule_ptr(cl, "zunglq")]
    lib.orc_set_lapack.argtypes = [ctypes.c_void_p] * 6
    if lib.orc_set_lapack(*ptrs) != 0:
        raise RuntimeError("oracle: missing BLAS/LAPACK entry points")
    P, I, D, U64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_uint64
    sig = {
        "orc_create": ([I, I, I, I, D, I], P),
        "orc_destroy": ([P], None),
        "orc_set_threads": ([P, I], None),
        "orc_set_spvn": ([P, I, I, P, P, P], None),
        "orc_set_spvnT": ([P, I, I, P, P, P], None),
        "orc_set_vakbl": ([P, I, I, P, P, P], None),
        "orc_set_dense": ([P, P, P, P, P], None),
        "orc_set_walkers": ([P, P, P], None),
        "orc_get_walkers": ([P, P, P], None),
        "orc_copy_out": ([P, I, P], None),
        "orc_get_eshift": ([P], D),
        "orc_set_eshift": ([P, D], None),
        "orc_mixed_density_matrix": ([P], None),
        "orc_overlaps": ([P, I], None),
        "orc_vbias": ([P], None),
        "orc_mixed_density_matrix_full": ([P], None),
        "orc_vbias_full": ([P], None),
        "orc_generate_x": ([P, U64, U64], None),
        "orc_sigma": ([P, U64, U64], None),
        "orc_sigma_from": ([P, P], None),
        "orc_vhs": ([P], None),
        "orc_propagate": ([P], None),
        "orc_update_weights": ([P], None),
        "orc_sum_e4": ([P], D),
        "orc_orthogonalize": ([P], None),
        "orc_energy_vakbl": ([P], D),
        "orc_energy_chol": ([P, P], D),
        "orc_halfrotate": ([I, I, I, P, P, P, P, P, D, P, P, P], ctypes.c_longlong),
        "orc_csrmm": ([ctypes.c_char, I, I, P, P, P, I, P, P, I, P, P, I], None),
        "orc_rm_gemm": ([ctypes.c_char, ctypes.c_char, I, I, I, P, I, P, I, P, I], None),
        "orc_invert": ([I, P, P], I),
        "orc_normals": ([U64, U64, ctypes.c_longlong, P], None),
        "orc_set_walker_offset": ([P, I, ctypes.c_longlong], None),
        "orc_philox": ([P, P, P], None),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _LIBS[path] = lib
    return lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def _c(a, dtype) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=dtype)


class Oracle:
    """Reference-structured FP64 CPU implementation of one walker ensemble.

    Methods mirror the reference's operation calls (afqmc_sys.hpp, vbias.hpp, vHS.hpp,
    energy.hpp) and the driver's inline steps (miniafqmc_base.cpp:281-327)."""

    def __init__(self, system, nwalk: int, fast: bool = False, threads: int = 1):
        self.lib = load(fast)
        self.sys = system
        N, n, nc = system.N, system.n, system.nchol
        self.N, self.n, self.nchol, self.nw = N, n, nc, nwalk
        self.h = self.lib.orc_create(N, n, nc, nwalk, system.cfg.dt, system.cfg.taylor_order)
        self.lib.orc_set_threads(self.h, threads)
        self._keep = []
        for fn, m in (("orc_set_spvn", system.Spvn), ("orc_set_spvnT", system.SpvnT),
                      ("orc_set_vakbl", system.Vakbl)):
            if m is None:
                continue
            ri, ci, v = _c(m.rowIndex, np.int32), _c(m.cols, np.int32), _c(m.vals, np.complex128)
            getattr(self.lib, fn)(self.h, m.nrows, m.ncols, _p(ri), _p(ci), _p(v))
        P = _c(system.Propg1, np.complex128)
        haj = _c(system.haj, np.complex128)
        tr = _c(system.trial, np.complex128)
        Lh = None if system.Lh is None else _c(system.Lh, np.complex128)
        self.lib.orc_set_dense(self.h, _p(P), _p(haj), _p(tr), None if Lh is None else _p(Lh))
        W, Wd = system.initial_walkers(nwalk)
        self.set_walkers(W, Wd)

    def __del__(self):
        try:
            self.lib.orc_destroy(self.h)
        except Exception:
            pass

    # state -------------------------------------------------------------------------
    def set_walkers(self, W, Wd):
        W, Wd = _c(W, np.complex128), _c(Wd, np.complex128)
        self.lib.orc_set_walkers(self.h, _p(W), _p(Wd))

    def get_walkers(self):
        W = np.empty((self.nw, 2, self.N, self.n), np.complex128)
        Wd = np.empty((self.nw, 8), np.complex128)
        self.lib.orc_get_walkers(self.h, _p(W), _p(Wd))
        return W, Wd

    def copy_out(self, which: str) -> np.ndarray:
        nw, N, n, nc = self.nw, self.N, self.n, self.nchol
        shapes = {"Gc": ((2 * n * N, nw), np.complex128, 0), "vbias": ((nc, nw), np.complex128, 1),
                  "X": ((nc, nw), np.complex128, 2), "vHS": ((N * N, nw), np.complex128, 3),
                  "hybridW": ((nw,), np.complex128, 4), "xraw": ((nc, nw), np.float64, 5),
                  "info": ((nw, 2), np.int32, 6), "G_full": ((2 * N * N, nw), np.complex128, 7)}
        shape, dt, code = shapes[which]
        out = np.empty(shape, dt)
        self.lib.orc_copy_out(self.h, code, _p(out))
        return out

    def set_walker_offset(self, offset: int, nwalk_global: int):
        self.lib.orc_set_walker_offset(self.h, offset, nwalk_global)
        self.walker_offset = offset

    @property
    def eshift(self) -> float:
        return self.lib.orc_get_eshift(self.h)

    @eshift.setter
    def eshift(self, v: float):
        self.lib.orc_set_eshift(self.h, float(v))

    # operations --------------------------------------------------------------------
    def calculate_mixed_density_matrix(self):
        self.lib.orc_mixed_density_matrix(self.h)

    def calculate_overlaps(self, save_old: bool = False):
        self.lib.orc_overlaps(self.h, int(save_old))

    def get_vbias(self):
        self.lib.orc_vbias(self.h)

    def calculate_mixed_density_matrix_full(self):
        """Non-compact density matrix G[2][N][N][nw] (transposed_Spvn == false)."""
        self.lib.orc_mixed_density_matrix_full(self.h)

    def get_vbias_full(self):
        """vbias = T(Spvn) G_alpha + T(Spvn) G_beta from the full density matrix."""
        self.lib.orc_vbias_full(self.h)

    def sigma(self, seed: int, step: int):
        self.lib.orc_sigma(self.h, seed, step)

    def sigma_from(self, x: np.ndarray):
        x = _c(x, np.float64)
        self.lib.orc_sigma_from(self.h, _p(x))

    def get_vHS(self):
        self.lib.orc_vhs(self.h)

    def propagate(self):
        self.lib.orc_propagate(self.h)

    def update_weights(self):
        self.lib.orc_update_weights(self.h)

    def sum_e4(self) -> float:
        return self.lib.orc_sum_e4(self.h)

    def update_weights_partial(self) -> float:
        """Weights with the current Eshift; returns the local sum of Re W_data[:,4]
        and leaves Eshift for the caller to set from the global sum."""
        e = self.eshift
        self.update_weights()
        self.eshift = e
        return self.sum_e4()

    def energy_sums(self, mode: str = "auto"):
        self.calculate_energy(mode)
        _, Wd = self.get_walkers()
        return np.array([np.sum(Wd[:, 0].real * Wd[:, 1].real), np.sum(Wd[:, 1].real)])

    def orthogonalize(self):
        self.lib.orc_orthogonalize(self.h)

    def population_control(self, seed: int, step: int):
        """The comb on this walker set (`comb` below), as afq_population_control."""
        W, Wd = self.get_walkers()
        Wn, Wdn, _ = comb(W, Wd, seed, step, getattr(self, "walker_offset", 0))
        self.set_walkers(Wn, Wdn)

    def calculate_energy(self, mode: str = "auto", parts: bool = False):
        if mode == "auto":
            mode = "vakbl" if self.sys.Vakbl is not None else "chol"
        if mode == "vakbl":
            return self.lib.orc_energy_vakbl(self.h)
        buf = np.zeros((self.nw, 3)) if parts else None
        e = self.lib.orc_energy_chol(self.h, None if buf is None else _p(buf))
        return (e, buf) if parts else e

    # the driver's substep (miniafqmc_base.cpp:251-337) ------------------------------
    def substep(self, seed: int, step_tot: int, northo: int, x: np.ndarray | None = None,
                graph: bool = False):
        self.calculate_mixed_density_matrix()
        self.get_vbias()
        if x is None:
            self.sigma(seed, step_tot)
        else:
            self.sigma_from(x)
        self.get_vHS()
        self.propagate()
        self.calculate_overlaps(save_old=True)
        self.update_weights()
        if step_tot > 0 and step_tot % northo == 0:
            self.orthogonalize()
            self.calculate_overlaps(save_old=False)


def normals(seed: int, step: int, count: int) -> np.ndarray:
    out = np.empty(count, np.float64)
    load().orc_normals(seed, step, count, _p(out))
    return out


def philox(ctr, key) -> np.ndarray:
    c = np.asarray(ctr, np.uint32)
    k = np.asarray(key, np.uint32)
    out = np.empty(4, np.uint32)
    load().orc_philox(_p(c), _p(k), _p(out))
    return out


def halfrotate(system, cutoff: float = 1e-6):
    """rotate.hpp:69-169 restated with zgemm; returns the CSR triple of SpvnT."""
    lib = load()
    S = system.Spvn
    ri, ci, v = _c(S.rowIndex, np.int32), _c(S.cols, np.int32), _c(S.vals, np.complex128)
    ta, tb = _c(system.trial[0], np.complex128), _c(system.trial[1], np.complex128)
    args = (system.N, system.n, system.nchol, _p(ri), _p(ci), _p(v), _p(ta), _p(tb), cutoff)
    nnz = lib.orc_halfrotate(*args, None, None, None)
    rowIndex = np.empty(system.nchol + 1, np.int32)
    cols = np.empty(nnz, np.int32)
    vals = np.empty(nnz, np.complex128)
    lib.orc_halfrotate(*args, _p(rowIndex), _p(cols), _p(vals))
    return rowIndex, cols, vals


# Population control by the comb (no reference counterpart: the reference leaves branching
# out, miniafqmc_base.cpp:347).  Weights w_i = max(Re W_data[i][1], 0), total T, prefix sums
# C_i in walker order; copy j takes the first walker with C_i > (j + u) T / nw and weight
# T / nw.  u is one Philox4x32-10 uniform for (seed, step, walker offset) on a key apart
# from the fields'; the blocks of a sharded ensemble comb on their own, each with the u of
# its offset (the global index of its first walker).
COMB_KEY = 0x9E3779B97F4A7C15


def comb_uniform(seed: int, step: int, offset: int = 0) -> float:
    key = (seed ^ COMB_KEY) & 0xFFFFFFFFFFFFFFFF
    c = philox([offset & 0xFFFFFFFF, 0, step & 0xFFFFFFFF, step >> 32],
               [key & 0xFFFFFFFF, key >> 32])
    c = [int(x) for x in c]
    return float(((c[0] >> 5) << 26) | (c[1] >> 6)) * (1.0 / 9007199254740992.0)


def comb(W: np.ndarray, Wd: np.ndarray, seed: int, step: int, offset: int = 0):
    """(new walkers, new walker data, parent index of each copy)."""
    nw = Wd.shape[0]
    w = np.maximum(Wd[:, 1].real, 0.0)
    if not np.any(w > 0):
        raise ValueError("population control: no walker has positive weight")
    C = np.cumsum(w)
    T = C[-1]
    u = comb_uniform(seed, step, offset)
    t = (np.arange(nw, dtype=np.float64) + u) * T / nw
    idx = np.searchsorted(C, t, side="right")
    last = int(np.nonzero(w > 0)[0][-1])
    idx = np.where(idx < nw, idx, last)
    Wn, Wdn = W[idx].copy(), Wd[idx].copy()
    Wdn[:, 1] = T / nw
    return Wn, Wdn, idx

