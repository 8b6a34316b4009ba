"""Host-side mirror of the miniapp's AFQMC operation interface over libafqmc_b200.

`AfqmcSys` carries the same operation names as the reference's `base::afqmc_sys` and
free functions (src/AFQMC/afqmc_sys.hpp, vbias.hpp, vHS.hpp, energy.hpp), but the walker
set lives on the GPU inside the handle; every call goes through the C ABI declared in
include/afqmc_b200.h.  Errors come back as `AfqmcError` carrying the library's status.

The library must be built (`python -m miniafqmc_b200.build`); there is no CPU
fallback, and loading fails loudly when the shared object is missing."""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libafqmc_b200.so")

AFQ_PREC_FP64, AFQ_PREC_MIXED = 0, 1
AFQ_ENERGY_VAKBL, AFQ_ENERGY_CHOLESKY, AFQ_ENERGY_CV = 0, 1, 2
BUFFERS = {"Gc": 0, "vbias": 1, "X": 2, "vHS": 3, "hybridW": 4, "xraw": 5, "info": 6,
           "energy_parts": 7, "cv_pred": 8, "G_full": 9}
STATUS = {0: "AFQ_OK", 1: "AFQ_ERR_ARG", 2: "AFQ_ERR_STATE", 3: "AFQ_ERR_CUDA",
          4: "AFQ_ERR_OOM", 5: "AFQ_ERR_UNSUPPORTED", 6: "AFQ_ERR_SINGULAR"}

EXPORTS = [
    "afq_create", "afq_destroy", "afq_status_string", "afq_last_error", "afq_set_hamiltonian",
    "afq_set_walkers", "afq_get_walkers", "afq_mixed_density_matrix", "afq_overlaps",
    "afq_vbias", "afq_sigma", "afq_sigma_from", "afq_vhs", "afq_propagate",
    "afq_update_weights", "afq_update_weights_partial", "afq_get_eshift", "afq_set_eshift",
    "afq_orthogonalize", "afq_energy", "afq_energy_sums", "afq_substep", "afq_synchronize",
    "afq_copy_out", "afq_set_walker_offset", "afq_profile", "afq_stage_times", "afq_get_stream",
    "afq_selftest_tc_gemm", "afq_exchange_energy_noalloc", "afq_cv_configure", "afq_cv_set_base", "afq_cv_stats",
    "afq_mlp_create", "afq_mlp_destroy", "afq_mlp_num_params", "afq_mlp_set_params",
    "afq_mlp_get_params", "afq_mlp_forward", "afq_mlp_gradient", "afq_mlp_train",
    "afq_batch_create", "afq_batch_destroy", "afq_batch_substep", "afq_batch_synchronize",
    "afq_get_tuning", "afq_halfrotate", "afq_population_control",
    "afq_mixed_density_matrix_full", "afq_vbias_full", "afq_get_sparse_paths",
    "afq_set_tc_wait_limit", "afq_substep_begin", "afq_substep_end", "afq_batch_substeps",
    "afq_copy_walkers", "afq_get_schedule", "afq_batch_set_fused",
]
STAGES = ["DM", "vbias", "sigma", "vHS", "propagate", "overlap", "weights", "ortho", "energy"]


class AfqmcError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class SystemDesc(ctypes.Structure):
    _fields_ = [("nmo", ctypes.c_int), ("naea", ctypes.c_int), ("naeb", ctypes.c_int),
                ("nchol", ctypes.c_int), ("nwalk", ctypes.c_int), ("dt", ctypes.c_double),
                ("taylor_order", ctypes.c_int), ("precision", ctypes.c_int),
                ("device", ctypes.c_int)]


class CsrZ(ctypes.Structure):
    _fields_ = [("nrows", ctypes.c_int), ("ncols", ctypes.c_int),
                ("rowIndex", ctypes.c_void_p), ("cols", ctypes.c_void_p),
                ("vals", ctypes.c_void_p)]


_LIB = None


def signatures() -> dict:
    """ctypes (argtypes, restype) of every entry point of include/afqmc_b200.h."""
    P, I, D, U64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_uint64
    return {
        "afq_create": ([P, P], I), "afq_destroy": ([P], None),
        "afq_status_string": ([I], ctypes.c_char_p), "afq_last_error": ([P], ctypes.c_char_p),
        "afq_set_hamiltonian": ([P, P, P, P, P, P, P, P], I),
        "afq_set_walkers": ([P, P, P], I), "afq_get_walkers": ([P, P, P], I),
        "afq_mixed_density_matrix": ([P], I), "afq_overlaps": ([P, I], I),
        "afq_vbias": ([P], I), "afq_sigma": ([P, U64, U64], I), "afq_sigma_from": ([P, P], I),
        "afq_vhs": ([P], I), "afq_propagate": ([P], I), "afq_update_weights": ([P], I),
        "afq_update_weights_partial": ([P, P], I), "afq_get_eshift": ([P, P], I),
        "afq_set_eshift": ([P, D], I), "afq_orthogonalize": ([P], I),
        "afq_energy": ([P, I, P], I), "afq_energy_sums": ([P, I, P], I),
        "afq_substep": ([P, U64, U64, I], I), "afq_synchronize": ([P], I),
        "afq_copy_out": ([P, I, P], I), "afq_set_walker_offset": ([P, I, I], I),
        "afq_profile": ([P, I], I), "afq_stage_times": ([P, P, P, I], I),
        "afq_get_stream": ([P, P], I),
        "afq_selftest_tc_gemm": ([I, I, I, I, I, I, I, P, P, P, P], I),
        "afq_exchange_energy_noalloc": ([P, P, I, I, I, I, P, P], I),
        "afq_cv_configure": ([P, I, D, U64, ctypes.c_longlong, I], I),
        "afq_cv_set_base": ([P, I], I),
        "afq_cv_stats": ([P, P], I),
        "afq_mlp_create": ([I, I, I, U64, P], I), "afq_mlp_destroy": ([P], None),
        "afq_mlp_num_params": ([P], ctypes.c_longlong), "afq_mlp_set_params": ([P, P], I),
        "afq_mlp_get_params": ([P, P], I), "afq_mlp_forward": ([P, I, P, P], I),
        "afq_mlp_gradient": ([P, I, P, P, P, P], I),
        "afq_mlp_train": ([P, I, P, P, I, ctypes.c_float, P], I),
        "afq_batch_create": ([P, I, P], I), "afq_batch_destroy": ([P], None),
        "afq_batch_substep": ([P, P, U64, I], I), "afq_batch_synchronize": ([P], I),
        "afq_get_tuning": ([P, P, P], I),
        "afq_halfrotate": ([I, P, I, I, I, P, D, D, P, P, P, P, P], I),
        "afq_population_control": ([P, U64, U64], I),
        "afq_mixed_density_matrix_full": ([P], I), "afq_vbias_full": ([P], I),
        "afq_get_sparse_paths": ([P, P, P], I),
        "afq_set_tc_wait_limit": ([I, ctypes.c_longlong], I),
        "afq_substep_begin": ([P, U64, U64, P], I), "afq_substep_end": ([P, U64, I], I),
        "afq_batch_substeps": ([P, P, U64, I, I], I),
        "afq_copy_walkers": ([P, P], I), "afq_get_schedule": ([P, P, P], I),
        "afq_batch_set_fused": ([P, I], I),
    }


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads the CUDA library; raises if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m miniafqmc_b200.build`")
    lib = ctypes.CDLL(path)
    for name, (args, res) in signatures().items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _LIB = lib
    return lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def _csr(m):
    if m is None:
        return None, ()
    ri = np.ascontiguousarray(m.rowIndex, np.int32)
    ci = np.ascontiguousarray(m.cols, np.int32)
    v = np.ascontiguousarray(m.vals, np.complex128)
    s = CsrZ(m.nrows, m.ncols, _p(ri), _p(ci), _p(v))
    return s, (ri, ci, v)


class AfqmcSys:
    """One device-resident walker set with its Hamiltonian (mirrors base::afqmc_sys)."""

    def __init__(self, system, nwalk: int, precision: int = AFQ_PREC_FP64, device: int = 0,
                 use_vakbl: bool = True, use_chol: bool = True, walkers=None):
        self.lib = load_library()
        self.sys = system
        self.N, self.n, self.nchol, self.nw = system.N, system.n, system.nchol, nwalk
        self.precision = precision
        desc = SystemDesc(system.N, system.n, system.n, system.nchol, nwalk, system.cfg.dt,
                          system.cfg.taylor_order, precision, device)
        h = ctypes.c_void_p()
        st = self.lib.afq_create(ctypes.byref(desc), ctypes.byref(h))
        if st != 0:
            raise AfqmcError(st, "afq_create failed")
        self.h = h
        sp, k1 = _csr(system.Spvn)
        spT, k2 = _csr(system.SpvnT)
        vk, k3 = _csr(system.Vakbl if use_vakbl else None)
        P = np.ascontiguousarray(system.Propg1, np.complex128)
        haj = np.ascontiguousarray(system.haj, np.complex128)
        tr = np.ascontiguousarray(system.trial, np.complex128)
        Lh = np.ascontiguousarray(system.Lh, np.complex128) if (use_chol and system.Lh is not None) else None
        self._check(self.lib.afq_set_hamiltonian(
            self.h, ctypes.byref(sp), ctypes.byref(spT), _p(P), _p(haj), _p(tr),
            ctypes.byref(vk) if vk is not None else None, _p(Lh) if Lh is not None else None))
        del k1, k2, k3
        self.has_vakbl = vk is not None
        self.has_chol = Lh is not None
        W, Wd = walkers if walkers is not None else system.initial_walkers(nwalk)
        self.set_walkers(W, Wd)

    def _check(self, st: int):
        if st != 0:
            msg = self.lib.afq_last_error(self.h)
            raise AfqmcError(st, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "h", None):
            self.lib.afq_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # state -------------------------------------------------------------------------
    def set_walkers(self, W, Wd):
        W = np.ascontiguousarray(W, np.complex128)
        Wd = np.ascontiguousarray(Wd, np.complex128)
        self._check(self.lib.afq_set_walkers(self.h, _p(W), _p(Wd)))

    def get_walkers(self):
        W = np.empty((self.nw, 2, self.N, self.n), np.complex128)
        Wd = np.empty((self.nw, 8), np.complex128)
        self._check(self.lib.afq_get_walkers(self.h, _p(W), _p(Wd)))
        return W, Wd

    def copy_walkers_from(self, other: "AfqmcSys"):
        """This handle's walkers := other's (device to device, afq_copy_walkers)."""
        self._check(self.lib.afq_copy_walkers(self.h, other.h))

    def get_walker_data(self):
        Wd = np.empty((self.nw, 8), np.complex128)
        self._check(self.lib.afq_get_walkers(self.h, None, _p(Wd)))
        return Wd

    def copy_out(self, which: str) -> np.ndarray:
        nw, N, n, nc = self.nw, self.N, self.n, self.nchol
        shapes = {"Gc": ((2 * n * N, nw), np.complex128), "vbias": ((nc, nw), np.complex128),
                  "X": ((nc, nw), np.complex128), "vHS": ((N * N, nw), np.complex128),
                  "hybridW": ((nw,), np.complex128), "xraw": ((nc, nw), np.float64),
                  "info": ((nw, 2), np.int32), "energy_parts": ((nw, 3), np.float64),
                  "cv_pred": ((nw,), np.float64), "G_full": ((2 * N * N, nw), np.complex128)}
        shape, dt = shapes[which]
        out = np.empty(shape, dt)
        self._check(self.lib.afq_copy_out(self.h, BUFFERS[which], _p(out)))
        return out

    @property
    def eshift(self) -> float:
        v = ctypes.c_double()
        self._check(self.lib.afq_get_eshift(self.h, ctypes.byref(v)))
        return v.value

    @eshift.setter
    def eshift(self, value: float):
        self._check(self.lib.afq_set_eshift(self.h, float(value)))

    # operations (reference names) ------------------------------------------------
    def calculate_mixed_density_matrix(self):
        self._check(self.lib.afq_mixed_density_matrix(self.h))

    def calculate_overlaps(self, save_old: bool = False):
        self._check(self.lib.afq_overlaps(self.h, int(save_old)))

    def get_vbias(self):
        self._check(self.lib.afq_vbias(self.h))

    def sigma(self, seed: int, step: int):
        self._check(self.lib.afq_sigma(self.h, seed, step))

    def sigma_from(self, x: np.ndarray):
        x = np.ascontiguousarray(x, np.float64)
        self._check(self.lib.afq_sigma_from(self.h, _p(x)))

    def get_vHS(self):
        self._check(self.lib.afq_vhs(self.h))

    def propagate(self):
        self._check(self.lib.afq_propagate(self.h))

    def update_weights(self):
        self._check(self.lib.afq_update_weights(self.h))

    def update_weights_partial(self) -> float:
        v = ctypes.c_double()
        self._check(self.lib.afq_update_weights_partial(self.h, ctypes.byref(v)))
        return v.value

    def orthogonalize(self):
        self._check(self.lib.afq_orthogonalize(self.h))

    def set_walker_offset(self, offset: int, nwalk_global: int):
        self._check(self.lib.afq_set_walker_offset(self.h, offset, nwalk_global))

    def calculate_energy(self, mode: str = "auto") -> float:
        m = self._mode(mode)
        v = ctypes.c_double()
        self._check(self.lib.afq_energy(self.h, m, ctypes.byref(v)))
        return v.value

    def energy_sums(self, mode: str = "auto"):
        m = self._mode(mode)
        buf = np.zeros(2)
        self._check(self.lib.afq_energy_sums(self.h, m, _p(buf)))
        return buf

    def _mode(self, mode: str) -> int:
        if mode == "auto":
            mode = "chol" if self.has_chol else "vakbl"
        return {"vakbl": AFQ_ENERGY_VAKBL, "chol": AFQ_ENERGY_CHOLESKY, "cv": AFQ_ENERGY_CV}[mode]

    def cv_configure(self, hidden: int = 256, lr: float = 1e-3, seed: int = 12345,
                     train_walker_steps: int = 2000, subset_den: int = 8):
        """Learned control variate for the exchange energy (used by mode "cv")."""
        self._check(self.lib.afq_cv_configure(self.h, hidden, lr, seed, train_walker_steps,
                                              subset_den))

    def cv_set_base(self, base: int = 1):
        """Two-level control variate: plain-bf16 exchange of every walker as the
        surrogate's base, the network learning the exact-minus-base residual (mixed form)."""
        self._check(self.lib.afq_cv_set_base(self.h, base))

    def cv_stats(self) -> dict:
        v = np.zeros(8)
        self._check(self.lib.afq_cv_stats(self.h, _p(v)))
        return {"samples": int(v[0]), "subset": int(v[1]), "loss": float(v[2]),
                "active": bool(v[3]), "measurements": int(v[4]), "subset_var": float(v[5]),
                "restandardisations": int(v[6]), "fallback": bool(v[7])}

    def calculate_mixed_density_matrix_full(self):
        """Full density matrix G[2][N][N] of every walker (the reference's -t no path)."""
        self._check(self.lib.afq_mixed_density_matrix_full(self.h))

    def get_vbias_full(self):
        """vbias = T(Spvn) G_alpha + T(Spvn) G_beta from the full density matrix."""
        self._check(self.lib.afq_vbias_full(self.h))

    def population_control(self, seed: int, step: int):
        """Comb resampling of the walkers (weights equalised, total weight kept)."""
        self._check(self.lib.afq_population_control(self.h, seed, step))

    TUNE_SITES = ["vhs", "propagate", "splitk", "exchange_all", "exchange_subset", "t1"]
    TUNE_SITES_FP64 = ["vhs_csr", "propagate_zgemm", "vbias_zgemm", "coulomb_zgemm",
                       "vakbl_zgemm"]

    def tuning(self) -> dict:
        """Kernels picked at set-up.  Mixed form: per tensor-core product site 0 (built-in
        rule), 1 (persistent) or 2 (per-tile) with the timed milliseconds of both
        candidates, and the split-K slice count.  FP64 form: per site the chosen CTA /
        tile shape index (0 = rule) with the milliseconds of the chosen shape and of the
        rule."""
        ns, nf = len(self.TUNE_SITES), len(self.TUNE_SITES_FP64)
        c = np.zeros(ns + 1 + nf, dtype=np.int32)
        t = np.zeros(2 * (ns + nf))
        self._check(self.lib.afq_get_tuning(self.h, _p(c), _p(t)))
        if self.precision != AFQ_PREC_MIXED:
            return {k: {"shape": int(c[ns + 1 + i]),
                        "ms": [round(float(t[2 * (ns + i)]), 4),
                               round(float(t[2 * (ns + i) + 1]), 4)]}
                    for i, k in enumerate(self.TUNE_SITES_FP64)}
        out = {k: {"kernel": int(c[i]), "ms": [round(float(t[2 * i]), 4),
                                               round(float(t[2 * i + 1]), 4)]}
               for i, k in enumerate(self.TUNE_SITES)}
        out["splitk_slices"] = int(c[ns])
        sc = np.zeros(3, np.int32)
        gm = np.zeros(16)
        self._check(self.lib.afq_get_schedule(self.h, _p(sc), _p(gm)))
        out["propagate_walker_group"] = {"walkers": int(sc[0]),
                                         "ms_all_32_48_64_96_128": [round(float(x), 4)
                                                                    for x in gm[:6]]}
        out["vhs_epilogue"] = {"tile": int(sc[1]),
                               "ms_rowwise_tile_tile2_tile2slab64": [round(float(x), 4)
                                                                     for x in gm[6:10]]}
        out["propagate_chain"] = {"wave": int(sc[2]),
                                  "ms_launches_16_24_32_48_64": [round(float(x), 4)
                                                                 for x in gm[10:16]]}
        return out

    SPARSE_OPERANDS = ["Spvn", "SpvnT", "Vakbl"]

    def sparse_paths(self) -> dict:
        """FP64 form: per sparse operand the product the set-up tuner kept ("dense",
        "csr", or None when absent) with the best milliseconds of the CSR and the dense
        product (0 when not timed)."""
        p = np.zeros(3, np.int32)
        t = np.zeros(6)
        self._check(self.lib.afq_get_sparse_paths(self.h, _p(p), _p(t)))
        names = {1: "dense", 0: "csr", -1: None}
        return {k: {"path": names[int(p[i])], "ms": [round(float(t[2 * i]), 4),
                                                      round(float(t[2 * i + 1]), 4)]}
                for i, k in enumerate(self.SPARSE_OPERANDS)}

    def substep(self, seed: int, step_tot: int, northo: int, graph: bool = True):
        """One substep of the driver loop (miniafqmc_base.cpp:251-337)."""
        if graph:
            self._check(self.lib.afq_substep(self.h, seed, step_tot, northo))
            return
        self.calculate_mixed_density_matrix()
        self.get_vbias()
        self.sigma(seed, step_tot)
        self.get_vHS()
        self.propagate()
        self.calculate_overlaps(save_old=True)
        self.update_weights()
        if step_tot > 0 and step_tot % northo == 0:
            self.orthogonalize()
            self.calculate_overlaps(save_old=False)

    def substep_begin(self, seed: int, step_tot: int) -> int:
        """First half of a walker-sharded substep (afq_substep_begin): returns the device
        address of the double holding this block's sum of Re W_data[:,4], which the caller
        all-reduces in place on the handle's stream before substep_end."""
        p = ctypes.c_void_p()
        self._check(self.lib.afq_substep_begin(self.h, seed, step_tot, ctypes.byref(p)))
        return p.value

    def substep_end(self, step_tot: int, northo: int):
        self._check(self.lib.afq_substep_end(self.h, step_tot, northo))

    def synchronize(self):
        self._check(self.lib.afq_synchronize(self.h))

    def profile(self, enable: bool = True):
        self._check(self.lib.afq_profile(self.h, int(enable)))

    def stage_times(self, reset: bool = True):
        """{stage: (gpu_ms, kernel_launches)} accumulated since the last reset."""
        ms = np.zeros(len(STAGES))
        nl = np.zeros(len(STAGES), np.int64)
        self._check(self.lib.afq_stage_times(self.h, _p(ms), _p(nl), int(reset)))
        return {k: (float(ms[i]), int(nl[i])) for i, k in enumerate(STAGES)}

    @property
    def stream(self) -> int:
        v = ctypes.c_void_p()
        self._check(self.lib.afq_get_stream(self.h, ctypes.byref(v)))
        return v.value or 0


def halfrotate(system, cutoff: float = 1e-6, device: int = 0, dense: bool = False):
    """GPU half-rotation of the system's Spvn with its trial (rotate.hpp:69-169): returns
    the SpvnT CSR triple (rowIndex, cols, vals) and, with dense=True, the unscaled dense
    factors Lh [nchol][2][n][N] as well."""
    lib = load_library()
    S = system.Spvn
    ri = np.ascontiguousarray(S.rowIndex, dtype=np.int32)
    ci = np.ascontiguousarray(S.cols, dtype=np.int32)
    v = np.ascontiguousarray(S.vals, dtype=np.complex128)
    keep = (ri, ci, v)
    m = CsrZ(S.nrows, S.ncols, _p(ri), _p(ci), _p(v))
    tr = np.ascontiguousarray(system.trial, dtype=np.complex128)
    N, n, nc = system.N, system.n, system.nchol
    nnz = ctypes.c_longlong()
    scale = 1.0 / np.sqrt(system.cfg.dt)
    args = (device, ctypes.byref(m), N, n, nc, _p(tr), cutoff, scale, ctypes.byref(nnz))
    st = lib.afq_halfrotate(*args, None, None, None, None)
    if st != 0:
        raise AfqmcError(st, "afq_halfrotate (count) failed")
    rowIndex = np.empty(nc + 1, np.int32)
    cols = np.empty(nnz.value, np.int32)
    vals = np.empty(nnz.value, np.complex128)
    Lh = np.empty((nc, 2, n, N), np.complex128) if dense else None
    st = lib.afq_halfrotate(*args, _p(rowIndex), _p(cols), _p(vals),
                            _p(Lh) if dense else None)
    if st != 0:
        raise AfqmcError(st, "afq_halfrotate failed")
    del keep
    return (rowIndex, cols, vals, Lh) if dense else (rowIndex, cols, vals)


class AfqmcBatch:
    """Several systems (AfqmcSys handles of any sizes, one device) advanced together:
    one CUDA-graph launch per substep, the systems' stages as parallel graph branches."""

    def __init__(self, systems):
        self.lib = load_library()
        self.systems = list(systems)
        arr = (ctypes.c_void_p * len(self.systems))(*[s.h for s in self.systems])
        self._arr = arr
        h = ctypes.c_void_p()
        st = self.lib.afq_batch_create(arr, len(self.systems), ctypes.byref(h))
        if st != 0:
            raise AfqmcError(st, "afq_batch_create failed")
        self.b = h

    def set_fused(self, fused=True):
        """Fused batch (afq_batch_set_fused): True (3) runs the vHS product and each
        propagation product as one launch over every system's tiles, 1 the vHS product
        only, 2 the propagation chain only, False (0) neither.  Raises AfqmcError when a
        system is not in the mixed form or the systems' precisions or Taylor orders
        differ."""
        mode = 3 if fused is True else 0 if fused is False else int(fused)
        st = self.lib.afq_batch_set_fused(self.b, mode)
        if st != 0:
            raise AfqmcError(st, "afq_batch_set_fused failed")

    def substep(self, seeds, step_tot: int, northo: int):
        sd = np.ascontiguousarray(seeds, dtype=np.uint64)
        st = self.lib.afq_batch_substep(self.b, _p(sd), step_tot, northo)
        if st != 0:
            raise AfqmcError(st, "afq_batch_substep failed")

    def substeps(self, seeds, step_tot: int, nsub: int, northo: int):
        """nsub substeps of every system in one graph launch (afq_batch_substeps)."""
        sd = np.ascontiguousarray(seeds, dtype=np.uint64)
        st = self.lib.afq_batch_substeps(self.b, _p(sd), step_tot, nsub, northo)
        if st != 0:
            raise AfqmcError(st, "afq_batch_substeps failed")

    def synchronize(self):
        st = self.lib.afq_batch_synchronize(self.b)
        if st != 0:
            raise AfqmcError(st, "afq_batch_synchronize failed")

    def close(self):
        if self.b:
            self.lib.afq_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Mlp:
    """The control variate's surrogate network on its own (afq_mlp_* entry points)."""

    def __init__(self, nin: int = 36, hidden: int = 256, capacity: int = 4096, seed: int = 1):
        self.lib = load_library()
        h = ctypes.c_void_p()
        st = self.lib.afq_mlp_create(nin, hidden, capacity, seed, ctypes.byref(h))
        if st != 0:
            raise AfqmcError(st, "afq_mlp_create failed")
        self.h, self.nin, self.hidden = h, nin, hidden
        self.nparams = int(self.lib.afq_mlp_num_params(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.lib.afq_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, st):
        if st != 0:
            raise AfqmcError(st, "mlp call failed")

    def get_params(self) -> np.ndarray:
        p = np.empty(self.nparams, np.float32)
        self._chk(self.lib.afq_mlp_get_params(self.h, _p(p)))
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        self._chk(self.lib.afq_mlp_set_params(self.h, _p(p)))

    def forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        y = np.empty(x.shape[0], np.float32)
        self._chk(self.lib.afq_mlp_forward(self.h, x.shape[0], _p(x), _p(y)))
        return y

    def gradient(self, x: np.ndarray, t: np.ndarray):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        g = np.empty(self.nparams, np.float32)
        loss = ctypes.c_float()
        self._chk(self.lib.afq_mlp_gradient(self.h, x.shape[0], _p(x), _p(t), _p(g),
                                            ctypes.byref(loss)))
        return g, loss.value

    def train(self, x: np.ndarray, t: np.ndarray, iters: int, lr: float = 1e-3) -> float:
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        loss = ctypes.c_float()
        self._chk(self.lib.afq_mlp_train(self.h, x.shape[0], _p(x), _p(t), iters, lr,
                                         ctypes.byref(loss)))
        return loss.value
