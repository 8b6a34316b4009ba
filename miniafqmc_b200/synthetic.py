"""Seeded synthetic closed-shell AFQMC systems in the miniapp's data layout.

The miniapp reads its Hamiltonian from HDF5 (`src/Matrix/initialize_serial.hpp:37-228`);
the datasets it reads are reproduced here as numpy arrays under the same names:

  /Wavefunctions/PureSingleDeterminant/{dims, hij, hij_indx, Wavefun,
                                        SpHijkl_vals, SpHijkl_cols, SpHijkl_rowIndex}
  /Propagators/phaseless_ImpSamp_ForceBias/{Spvn_dims, Spvn_propg1, Spvn_block_sizes,
                                            Spvn_index_0, Spvn_vals_0}

and `System.initialize()` turns them into the in-memory objects that `afqmc::Initialize`
plus `base::halfrotate_cholesky` leave behind (`miniafqmc_base.cpp:176-185`):

  Spvn   CSR [NMO^2 x nchol], values scaled by sqrt(dt)      (initialize_serial.hpp:197-221)
  SpvnT  CSR [nchol x 2*NAEA*NMO], half-rotated, |v|>1e-6    (rotate.hpp:69-169)
  trial  conj(Wavefun), alpha and beta blocks [NMO][NAEA]    (initialize_serial.hpp:113-130)
  haj    [2*NAEA][NMO] half-rotated one-body matrix          (initialize_serial.hpp:89-108)
  Propg1 [NMO][NMO]                                          (initialize_serial.hpp:186-194)
  Vakbl  CSR [2*NAEA*NMO]^2 half-rotated two-body matrix     (initialize_serial.hpp:134-164)

System model (all configs): h1 = sym(N(0,0.1)) + diag(linspace(-2,2,N)); nchol real
symmetric Cholesky vectors L_n with the requested fraction of nonzeros drawn
N(0, sigma), sigma = 0.05 at NMO=64/nchol=256/10% and size-scaled (Config.sigma);
trial = the lowest NAEA eigenvectors of h1 for both spins; Propg1 =
expm(-dt/2 (h1 - 1/2 sum_n L_n L_n)).  Everything is drawn from numpy's Philox
bit generator seeded with `seed`.

The two-body matrix follows the definition in `src/AFQMC/energy.hpp:37-51`:
  V[(s,a,k),(s',b,l)] = sum_ij tw_s(i,a) tw_s'(j,b) [(ik|jl) - d_ss' (il|jk)],
  (ik|jl) = sum_n L_n(i,k) L_n(j,l)
with L unscaled, so that 1/2 Gc.V.Gc equals the Coulomb-minus-exchange energy built from
the unscaled half-rotated factors Lh_s[n][a][k] = sum_i tw_s(i,a) L_n(i,k).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np
import scipy.linalg
import scipy.sparse as sp

HALFROTATE_CUTOFF = 1e-6  # rotate.hpp:69 default cutoff
INPUT_MAGIC = b"AFQINP01"  # the driver binary's input file (System.write_input)


@dataclasses.dataclass
class CSR:
    """Zero-based CSR triple with int32 indices and complex128 values.

    Rows sorted, columns sorted within a row, as `SparseMatrix::compress`
    leaves them (`src/Matrix/SparseMatrix.hpp:295-319`)."""
    nrows: int
    ncols: int
    rowIndex: np.ndarray  # int32 [nrows+1]
    cols: np.ndarray      # int32 [nnz]
    vals: np.ndarray      # complex128 [nnz]

    @property
    def nnz(self) -> int:
        return int(self.cols.shape[0])

    @classmethod
    def from_scipy(cls, m) -> "CSR":
        m = sp.csr_matrix(m)
        m.sum_duplicates()
        m.sort_indices()
        return cls(m.shape[0], m.shape[1], m.indptr.astype(np.int32),
                   m.indices.astype(np.int32), m.data.astype(np.complex128))

    def to_scipy(self):
        return sp.csr_matrix((self.vals, self.cols, self.rowIndex),
                             shape=(self.nrows, self.ncols))

    def todense(self) -> np.ndarray:
        return self.to_scipy().toarray()

    def density(self) -> float:
        return self.nnz / float(self.nrows * self.ncols)


@dataclasses.dataclass
class Config:
    nmo: int
    nel: int          # NAEA == NAEB
    nchol: int
    density: float
    seed: int
    dt: float = 0.005
    nwalk: int = 16
    nsteps: int = 20
    northo: int = 5
    energy_every: int = 1
    taylor_order: int = 6
    with_vakbl: bool = True
    complex_trial: bool = False   # rotate the trial by a random unitary (tests conj paths)
    complex_chol: bool = False    # give the Cholesky vectors an imaginary part
    chol_sigma: float | None = None  # std of the nonzeros (default: size-scaled, see below)

    @property
    def sigma(self) -> float:
        """Standard deviation of the Cholesky nonzeros: 0.05 at the 64-orbital,
        256-vector, 10%-dense system, scaled by sqrt(64*256*0.1 / (nmo*nchol*density))
        elsewhere so the two-body diagonal sum_n L_n(i,k)^2 is the same at every size
        (with a fixed 0.05 it grows ~70x at NMO=384, nchol=1536, 20% and the propagator
        becomes unstable: overlaps overflow within a few substeps)."""
        if self.chol_sigma is not None:
            return self.chol_sigma
        return 0.05 * math.sqrt(64 * 256 * 0.1 / (self.nmo * self.nchol * self.density))

    @property
    def name(self) -> str:
        return (f"NMO{self.nmo}_N{self.nel}_nchol{self.nchol}_d{self.density:g}"
                f"_W{self.nwalk}_seed{self.seed}")


# The workload table: C1 and C2 are the parity-test cases, C3 (Spvn above the dense
# threshold) and C4 run through `bench.py --config`, C4 is the bench's default workload and
# C5 the heterogeneous batch.
CONFIGS = {
    # small closed shell, every stage checked against the FP64 oracle
    "C1": Config(64, 16, 256, 0.10, 0, dt=0.005, nwalk=16, nsteps=20, northo=5,
                 energy_every=1),
    # batched FP64, one launch per stage, graph per step
    "C2": Config(128, 32, 512, 0.05, 1, dt=0.005, nwalk=256, nsteps=100, northo=5,
                 energy_every=2),
    # mixed precision, dense-tile path
    "C3": Config(256, 64, 1024, 0.30, 2, dt=0.005, nwalk=512, nsteps=200, northo=5,
                 energy_every=10, with_vakbl=False),
    # target configuration: NMO=384, 48+48 electrons, nchol=1536, 1024 walkers
    "C4": Config(384, 48, 1536, 0.20, 3, dt=0.005, nwalk=1024, nsteps=500, northo=5,
                 energy_every=10, with_vakbl=False),
}

# heterogeneous batch: three systems of uneven size advanced together (AfqmcBatch)
C5_SYSTEMS = [
    Config(96, 12, 384, 0.10, 4, dt=0.005, nwalk=128, nsteps=300, northo=5, energy_every=10,
           with_vakbl=False),
    Config(200, 40, 800, 0.10, 5, dt=0.005, nwalk=256, nsteps=300, northo=5, energy_every=10,
           with_vakbl=False),
    Config(320, 64, 1280, 0.10, 6, dt=0.005, nwalk=384, nsteps=300, northo=5, energy_every=10,
           with_vakbl=False),
]


def _sym_chol_coo(rng, N: int, nchol: int, density: float, complex_chol: bool,
                  sigma: float = 0.05):
    """COO (row = i*N+k, col = n, value) of nchol symmetric N x N matrices."""
    iu, ju = np.triu_indices(N)
    npos = iu.shape[0]
    rows, cols, vals = [], [], []
    chunk = max(1, int(2e7 // npos))
    for n0 in range(0, nchol, chunk):
        n1 = min(nchol, n0 + chunk)
        mask = rng.random((n1 - n0, npos)) < density
        vec, pos = np.nonzero(mask)
        v = rng.normal(0.0, sigma, vec.shape[0])
        if complex_chol:
            v = v + 1j * rng.normal(0.0, 0.02, vec.shape[0])
        i, k = iu[pos], ju[pos]
        off = i != k
        rows.append((i * N + k).astype(np.int64))
        cols.append((vec + n0).astype(np.int64))
        vals.append(v)
        rows.append((k[off] * N + i[off]).astype(np.int64))
        cols.append((vec[off] + n0).astype(np.int64))
        vals.append(v[off])
    return (np.concatenate(rows), np.concatenate(cols),
            np.concatenate(vals).astype(np.complex128))


def halfrotate(trial_a: np.ndarray, trial_b: np.ndarray, L, cutoff: float | None):
    """Dense half-rotated factors, the product `rotate.hpp:116,122` forms per vector.

    Returns Lh[nchol][2][n][N] with Lh[c][s][a][k] = sum_i trial_s(i,a) L_c(i,k),
    L given as a scipy CSR [N^2 x nchol] with rows i*N+k.  When `cutoff` is not None,
    entries with |value| <= cutoff are set to zero (rotate.hpp:119,156)."""
    N, n = trial_a.shape
    nchol = L.shape[1]
    coo = sp.coo_matrix(L)
    i = coo.row // N
    k = coo.row % N
    # L2[i][k*nchol + c] = L_c(i,k)
    L2 = sp.csr_matrix((coo.data, (i, k * nchol + coo.col)), shape=(N, N * nchol))
    out = np.empty((nchol, 2, n, N), dtype=np.complex128)
    L2T = L2.T.tocsr()
    for s, t in enumerate((trial_a, trial_b)):
        if s == 1 and np.array_equal(trial_a, trial_b):
            out[:, 1] = out[:, 0]
            break
        # C[(k*nchol+c)][a] = sum_i L2[i][k*nchol+c] t[i][a]
        C = np.asarray(L2T @ t)               # [N*nchol][n]
        out[:, s] = C.reshape(N, nchol, n).transpose(1, 2, 0)
    if cutoff is not None:
        out[np.abs(out) <= cutoff] = 0.0
    return out


@dataclasses.dataclass
class System:
    cfg: Config
    # file-level data (the HDF5 datasets, see module docstring)
    h1: np.ndarray
    Wavefun: np.ndarray        # [2][N][n]
    spvn_coo: tuple            # (rows, cols, vals), unscaled
    Propg1: np.ndarray         # [N][N]
    # in-memory data after Initialize + halfrotate
    Spvn: CSR = None           # scaled by sqrt(dt)
    SpvnT: CSR = None          # [nchol][2nN]
    trial: np.ndarray = None   # [2][N][n] = conj(Wavefun)
    haj: np.ndarray = None     # [2n][N]
    Vakbl: CSR | None = None   # [2nN][2nN]
    Lh: np.ndarray = None      # [nchol][2][n][N] unscaled, no cutoff

    @property
    def N(self):
        return self.cfg.nmo

    @property
    def n(self):
        return self.cfg.nel

    @property
    def nchol(self):
        return self.cfg.nchol

    def hdf5_datasets(self) -> dict:
        """The datasets `afqmc::Initialize` reads, keyed by their HDF5 paths."""
        N, n = self.N, self.n
        wf = "/Wavefunctions/PureSingleDeterminant/"
        pr = "/Propagators/phaseless_ImpSamp_ForceBias/"
        # hij rows: alpha rows a in [0,n), beta rows N+a (initialize_serial.hpp:97-107)
        ai = np.arange(n)
        rows = np.concatenate([ai, N + ai])
        idx = (rows[:, None] * N + np.arange(N)[None, :]).reshape(-1).astype(np.int32)
        d = {
            wf + "hij_indx": idx,
            wf + "hij": self.haj.reshape(-1).astype(np.complex128),
            wf + "Wavefun": self.Wavefun.reshape(-1),
        }
        if self.Vakbl is not None:
            # file rows/cols use the spin-offset orbital space i*N+j with i in [0,2N)
            def unmap(lin):
                a, j = lin // N, lin % N
                i = np.where(a < n, a, a - n + N)
                return (i * N + j).astype(np.int32)
            V = self.Vakbl.to_scipy().tocoo()
            fr, fc = unmap(V.row), unmap(V.col)
            Vf = sp.csr_matrix((V.data, (fr, fc)), shape=(2 * N * N, 2 * N * N))
            Vf.sort_indices()
            d[wf + "SpHijkl_vals"] = Vf.data.astype(np.complex128)
            d[wf + "SpHijkl_cols"] = Vf.indices.astype(np.int32)
            d[wf + "SpHijkl_rowIndex"] = Vf.indptr.astype(np.int32)
            nnzv = Vf.nnz
        else:
            nnzv = 0
        d[wf + "dims"] = np.array([0, nnzv, 2 * N * N, 2 * N * N, N, n, n, 0], np.int32)
        r, c, v = self.spvn_coo
        d[pr + "Spvn_dims"] = np.array([r.shape[0], N * N, self.nchol, N, 1], np.int64)
        d[pr + "Spvn_propg1"] = self.Propg1.reshape(-1).astype(np.complex128)
        d[pr + "Spvn_block_sizes"] = np.array([r.shape[0]], np.int32)
        d[pr + "Spvn_index_0"] = np.stack([r, c], axis=1).reshape(-1).astype(np.int32)
        d[pr + "Spvn_vals_0"] = v
        return d

    def write_input(self, path: str) -> None:
        """The driver binary's input file (`miniafqmc_b200/miniafqmc -f path`): the
        in-memory data `afqmc::Initialize` leaves behind (initialize_serial.hpp:89-221),
        in place of the HDF5 file no library here can write.  Little-endian binary:

          char[8]  "AFQINP01"
          int32    nmo, naea, naeb, nchol
          float64  dt                        (the time step Propg1 was formed with)
          int32    has_vakbl
          CSR      Spvn [nmo^2 x nchol], values scaled by sqrt(dt)
          float64  Propg1 [nmo][nmo] complex
          float64  haj [2 naea][nmo] complex
          float64  trial [2][nmo][naea] complex  (conj(Wavefun))
          CSR      Vakbl [2 naea nmo]^2      (when has_vakbl)

        with CSR = int32 nrows, ncols; int64 nnz; int32 rowIndex[nrows+1];
        int32 cols[nnz]; float64 vals[nnz] complex.  The driver half-rotates Spvn
        itself, as the miniapp's main does (miniafqmc_base.cpp:181-185)."""
        def csr(f, m: CSR):
            f.write(np.array([m.nrows, m.ncols], "<i4").tobytes())
            f.write(np.array([m.nnz], "<i8").tobytes())
            f.write(np.ascontiguousarray(m.rowIndex, "<i4").tobytes())
            f.write(np.ascontiguousarray(m.cols, "<i4").tobytes())
            f.write(np.ascontiguousarray(m.vals, "<c16").tobytes())
        with open(path, "wb") as f:
            f.write(INPUT_MAGIC)
            f.write(np.array([self.N, self.n, self.n, self.nchol], "<i4").tobytes())
            f.write(np.array([self.cfg.dt], "<f8").tobytes())
            f.write(np.array([1 if self.Vakbl is not None else 0], "<i4").tobytes())
            csr(f, self.Spvn)
            for a in (self.Propg1, self.haj, self.trial):
                f.write(np.ascontiguousarray(a, "<c16").tobytes())
            if self.Vakbl is not None:
                csr(f, self.Vakbl)

    def initial_walkers(self, nwalk: int):
        """W[nw][2][N][n] = conj(trialwfn) and W_data with weight 1
        (miniafqmc_base.cpp:222-236)."""
        W = np.empty((nwalk, 2, self.N, self.n), np.complex128)
        W[:] = np.conj(self.trial)[None]
        Wd = np.zeros((nwalk, 8), np.complex128)
        Wd[:, 1] = 1.0
        return W, Wd


def read_input(path: str) -> dict:
    """The arrays of a `System.write_input` file (the driver binary's input)."""
    buf = open(path, "rb").read()
    pos = 0

    def take(dtype, count):
        nonlocal pos
        a = np.frombuffer(buf, dtype, count, pos)
        pos += a.nbytes
        return a

    def csr():
        nr, nc = (int(v) for v in take("<i4", 2))
        nnz = int(take("<i8", 1)[0])
        return CSR(nr, nc, take("<i4", nr + 1).copy(), take("<i4", nnz).copy(),
                   take("<c16", nnz).copy())

    if buf[:8] != INPUT_MAGIC:
        raise ValueError(f"{path}: not a driver input file")
    pos = 8
    nmo, naea, naeb, nchol = (int(v) for v in take("<i4", 4))
    dt = float(take("<f8", 1)[0])
    has_vakbl = int(take("<i4", 1)[0])
    d = {"nmo": nmo, "naea": naea, "naeb": naeb, "nchol": nchol, "dt": dt, "Spvn": csr()}
    d["Propg1"] = take("<c16", nmo * nmo).reshape(nmo, nmo).copy()
    d["haj"] = take("<c16", 2 * naea * nmo).reshape(2 * naea, nmo).copy()
    d["trial"] = take("<c16", 2 * nmo * naea).reshape(2, nmo, naea).copy()
    d["Vakbl"] = csr() if has_vakbl else None
    if pos != len(buf):
        raise ValueError(f"{path}: {len(buf) - pos} trailing bytes")
    return d


def make_system(cfg: Config, build_vakbl: bool | None = None) -> System:
    N, n, nchol = cfg.nmo, cfg.nel, cfg.nchol
    rng = np.random.Generator(np.random.Philox(cfg.seed))
    A = rng.normal(0.0, 0.1, (N, N))
    h1 = 0.5 * (A + A.T) + np.diag(np.linspace(-2.0, 2.0, N))
    rows, cols, vals = _sym_chol_coo(rng, N, nchol, cfg.density, cfg.complex_chol, cfg.sigma)
    evals, evecs = np.linalg.eigh(h1)
    wf = evecs[:, :n].astype(np.complex128)
    if cfg.complex_trial:
        Z = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
        U, _ = np.linalg.qr(Z)
        wf = wf @ U
    Wavefun = np.stack([wf, wf.copy()])
    # one-body propagator exp(-dt/2 (h1 - 1/2 sum_n L_n L_n))
    # sum_n L_n L_n = sum_n sum_k L_n(i,k) L_n(k,j); with L_n symmetric this is
    # sum over (n,k) of L_n(i,k) L_n(j,k), accumulated densely in blocks of vectors
    LL = np.zeros((N, N), dtype=np.complex128 if cfg.complex_chol else np.float64)
    order = np.argsort(cols, kind="stable")
    rs, cs, vs = rows[order], cols[order], vals[order]
    if not cfg.complex_chol:
        vs = vs.real
    bounds = np.searchsorted(cs, np.arange(0, nchol + 1))
    blk = max(1, int(4e6 // (N * N)))
    for c0 in range(0, nchol, blk):
        c1 = min(nchol, c0 + blk)
        lo, hi = bounds[c0], bounds[c1]
        D = np.zeros((N, (c1 - c0) * N), dtype=LL.dtype)
        r = rs[lo:hi]
        D[r // N, (cs[lo:hi] - c0) * N + r % N] = vs[lo:hi]
        LL += D @ D.T
    Propg1 = scipy.linalg.expm(-0.5 * cfg.dt * (h1 - 0.5 * LL)).astype(np.complex128)
    sysm = System(cfg=cfg, h1=h1, Wavefun=Wavefun, spvn_coo=(rows, cols, vals),
                  Propg1=Propg1)
    _initialize(sysm, cfg.with_vakbl if build_vakbl is None else build_vakbl)
    return sysm


def _initialize(s: System, build_vakbl: bool):
    cfg = s.cfg
    N, n, nchol = cfg.nmo, cfg.nel, cfg.nchol
    rows, cols, vals = s.spvn_coo
    L = sp.csr_matrix((vals, (rows, cols)), shape=(N * N, nchol))
    L.sum_duplicates()
    L.sort_indices()
    s.trial = np.conj(s.Wavefun)                               # initialize_serial.hpp:124,129
    sq = math.sqrt(cfg.dt)
    Ls = L * sq                                                # initialize_serial.hpp:221
    s.Spvn = CSR.from_scipy(Ls)
    # unscaled, uncut factors for the Cholesky energy
    s.Lh = halfrotate(s.trial[0], s.trial[1], L, None)
    # half-rotation of the scaled matrix with the 1e-6 cutoff (rotate.hpp:69-169);
    # sqrt(dt) * (trial^T L) equals trial^T (sqrt(dt) L) up to one rounding
    Lh_scaled = s.Lh * sq
    Lh_scaled[np.abs(Lh_scaled) <= HALFROTATE_CUTOFF] = 0.0
    s.SpvnT = CSR.from_scipy(sp.csr_matrix(Lh_scaled.reshape(nchol, 2 * n * N)))
    del Lh_scaled
    # haj(s*n+a, k) = sum_i tw_s(i,a) h1(i,k)
    haj = np.concatenate([s.trial[0].T @ s.h1, s.trial[1].T @ s.h1], axis=0)
    s.haj = haj.astype(np.complex128)
    if build_vakbl:
        s.Vakbl = build_vakbl_from_factors(s.Lh)


def build_vakbl_from_factors(Lh: np.ndarray) -> CSR:
    """V[(s,a,k),(s',b,l)] = sum_n Lh_s[n][a][k] Lh_s'[n][b][l]
                             - d_ss' sum_n Lh_s[n][a][l] Lh_s[n][b][k]."""
    nchol, _, n, N = Lh.shape
    F = Lh.reshape(nchol, 2 * n * N)
    V = F.T @ F                                        # Coulomb part
    for s in range(2):
        Fs = Lh[:, s]                                  # [nchol][a][k]
        # X[(a,k),(b,l)] = sum_n Fs[n][a][l] Fs[n][b][k]
        X = np.einsum("nal,nbk->akbl", Fs, Fs, optimize=True).reshape(n * N, n * N)
        sl = slice(s * n * N, (s + 1) * n * N)
        V[sl, sl] -= X
    return CSR.from_scipy(sp.csr_matrix(V))
